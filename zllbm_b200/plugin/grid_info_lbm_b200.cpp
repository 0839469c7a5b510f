// GridInfoLbmB200 and B200Session: see grid_info_lbm_b200.h.
#include "grid_info_lbm_b200.h"
#include <algorithm>
#include <string>
#include "collision_model/lbm_collision_models.h"
#include "criterion/criterion_manager.h"
#include "grid/grid_manager.h"
#include "immersed_boundary/immersed_boundary.h"
#include "io/log_write.h"

namespace rootproject {
namespace zllbm {

namespace {

int zl_bc_kind(lbmproject::ELbmBoundaryConditionScheme scheme) {
    switch (scheme) {
        case lbmproject::ELbmBoundaryConditionScheme::kBounceBack: return ZL_BC_BOUNCE_BACK;
        case lbmproject::ELbmBoundaryConditionScheme::kPeriodic: return ZL_BC_PERIODIC;
        case lbmproject::ELbmBoundaryConditionScheme::kNonEqExtrapolation: return ZL_BC_NONEQ_EXTRAPOLATION;
        default: return ZL_BC_NONE;
    }
}

std::vector<uint64_t> sorted_codes(const DefMap<DefInt>& layer) {
    std::vector<uint64_t> out;
    out.reserve(layer.size());
    for (const auto& it : layer) out.push_back(it.first.to_ullong());
    std::sort(out.begin(), out.end());
    return out;
}

// codes of layers[first], layers[first + 1], ..., layers[last] (clamped to the layers present)
void add_layers(const std::vector<DefMap<DefInt>>& layers, std::size_t first, std::size_t last,
                std::vector<uint64_t>* out) {
    for (std::size_t i = first; i < layers.size() && i <= last; ++i) {
        std::vector<uint64_t> c = sorted_codes(layers[i]);
        out->insert(out->end(), c.begin(), c.end());
    }
}

void unique_sorted(std::vector<uint64_t>* v) {
    std::sort(v->begin(), v->end());
    v->erase(std::unique(v->begin(), v->end()), v->end());
}

}  // namespace

B200Session::~B200Session() {
    if (ctx_) zl_destroy(ctx_);
}

void B200Session::Check(int rc) const {
    if (rc == ZL_OK) return;
    char msg[512] = "context creation failed (no usable CUDA device, or an invalid configuration)";
    if (ctx_) zl_last_error(ctx_, msg, sizeof(msg));
    amrproject::LogManager::LogError("zllbm_b200 (code " + std::to_string(rc) + "): " + msg);
}

void B200Session::Install(lbmproject::SolverLbmInterface* solver) {
    if (zl_abi_version() != ZL_ABI_VERSION)
        amrproject::LogManager::LogError("libzllbm_b200.so does not match the zllbm_b200.h it was built against");
    solver->ptr_grid_info_creator_ = std::make_unique<GridInfoLbmB200Creator>(this);
}

void B200Session::EnsureUploaded(const amrproject::GridManagerInterface& gm,
                                 const lbmproject::SolverLbmInterface& solver,
                                 const amrproject::CriterionManager* cm) {
    if (ctx_) return;
    const int dims = solver.GetSolverDim();
    const int q = solver.k0NumQ_;
    const int levels = static_cast<int>(gm.vec_ptr_grid_info_.size());
    // the values the application set on the solver and the grid manager (zl_config mirrors them)
    zl_config cfg{};
    cfg.lattice = dims == 2 ? ZL_D2Q9 : ZL_D3Q19;
    const bool mrt = dynamic_cast<const lbmproject::LbmMrtCollisionOpt*>(&solver.GetCollisionOperator(0)) != nullptr;
    for (int l = 1; l < levels; ++l) {
        const bool m = dynamic_cast<const lbmproject::LbmMrtCollisionOpt*>(&solver.GetCollisionOperator(l)) != nullptr;
        if (m != mrt) amrproject::LogManager::LogError("zllbm_b200: one collision operator for every level");
    }
    cfg.collision = mrt ? ZL_MRT : ZL_SRT;
    cfg.storage = options_.storage;
    cfg.max_level = gm.GetMaxLevel();
    cfg.viscosity = solver.GetDefaultViscosity();
    cfg.rho0 = solver.GetDefaultDensity();
    const auto& grid0 = dynamic_cast<const lbmproject::GridInfoLbmInteface&>(*gm.vec_ptr_grid_info_.at(0));
    for (const auto& [dir, bc] : grid0.domain_boundary_condition_) {
        const int face = static_cast<int>(dir) - 1;  // EDomainBoundaryDirection: kBoundaryXMin = 1
        if (face < 0 || face >= 6) continue;
        cfg.bc_kind[face] = zl_bc_kind(bc->boundary_scheme_);
        auto v = options_.boundary_values.find(dir);
        if (v != options_.boundary_values.end())
            for (std::size_t a = 0; a < v->second.size() && a < 3; ++a) cfg.bc_velocity[face][a] = v->second[a];
    }
    const auto lo = gm.GetMinIndexOfBackgroundNodeArrAsVec();
    const auto hi = gm.GetMaxIndexOfBackgroundNodeArrAsVec();
    for (int a = 0; a < dims; ++a) {
        cfg.domain_min[a] = static_cast<int32_t>(lo[a]);
        cfg.domain_max[a] = static_cast<int32_t>(hi[a]);
    }
    const auto& vel = solver.GetDefaultVelocity();
    for (std::size_t a = 0; a < vel.size() && a < 3; ++a) cfg.init_velocity[a] = vel[a];
    cfg.forcing = solver.GetNumForces() > 0 ? 1 : 0;
    const auto& cf = solver.GetConstantForce();
    for (std::size_t a = 0; a < cf.size() && a < 3; ++a) cfg.constant_force[a] = cf[a];
    cfg.les = options_.les ? ZL_LES_SMAGORINSKY : 0;
    cfg.les_cs = options_.les_cs;
    cfg.dx = gm.GetDomainGridSize().at(0);
    cfg.device = options_.device;
    Check(zl_create(&cfg, &ctx_));

    // every level: node codes in the map's order and f_
    codes_.assign(levels, {});
    for (int l = 0; l < levels; ++l) {
        auto& grid = dynamic_cast<lbmproject::GridInfoLbmInteface&>(*gm.vec_ptr_grid_info_.at(l));
        auto& nodes = *grid.GetPtrToLbmGrid();
        std::vector<uint64_t>& codes = codes_[l];
        std::vector<double> f;
        codes.reserve(nodes.size());
        f.reserve(nodes.size() * q);
        for (const auto& [code, node] : nodes) {
            codes.push_back(code.to_ullong());
            f.insert(f.end(), node->f_.begin(), node->f_.end());
        }
        const auto n = static_cast<int64_t>(codes.size());
        Check(zl_set_level_nodes(ctx_, l, codes.data(), n));
        Check(zl_set_populations(ctx_, l, nullptr, f.data(), n));
    }
    // coarse/fine interfaces: the fine level's fine-to-coarse layers 1 and 2 are the explosion targets,
    // the coarse level's coarse-to-fine layer 1 the coalescence targets, its coarse-to-fine ghosts
    // are not explosion sources
    for (int l = 1; l < levels; ++l) {
        const auto& fine = *gm.vec_ptr_grid_info_.at(l);
        const auto& coarse = dynamic_cast<lbmproject::GridInfoLbmInteface&>(*gm.vec_ptr_grid_info_.at(l - 1));
        std::vector<uint64_t> c2f, f2c, ghost;
        for (const auto& [key, info] : fine.map_ptr_interface_layer_info_) {
            add_layers(info->vec_inner_fine2coarse_, 1, 2, &c2f);
            add_layers(info->vec_outer_fine2coarse_, 1, 2, &c2f);
        }
        for (const auto& [key, info] : coarse.map_ptr_interface_layer_info_) {
            add_layers(info->vec_inner_coarse2fine_, 1, 1, &f2c);
            add_layers(info->vec_outer_coarse2fine_, 1, 1, &f2c);
        }
        auto& cnodes = *const_cast<lbmproject::GridInfoLbmInteface&>(coarse).GetPtrToLbmGrid();
        for (const auto& [code, node] : cnodes)
            if (node->flag_status_ & amrproject::NodeBitStatus::kNodeStatusCoarse2FineGhost_)
                ghost.push_back(code.to_ullong());
        unique_sorted(&c2f);
        unique_sorted(&f2c);
        unique_sorted(&ghost);
        Check(zl_set_level_interface(ctx_, l, c2f.data(), static_cast<int64_t>(c2f.size()), f2c.data(),
                                     static_cast<int64_t>(f2c.size()), ghost.data(),
                                     static_cast<int64_t>(ghost.size())));
    }
    // immersed boundaries: the vertices of each geometry on its level, in key order
    if (cm) {
        for (const auto& geo : cm->vec_ptr_geometries_) {
            auto* ib = dynamic_cast<const lbmproject::GeometryInfoImmersedBoundary*>(geo.get());
            if (!ib) continue;
            std::vector<std::pair<DefSizet, const lbmproject::GeometryVertexImmersedBoundary*>> vs;
            for (const auto& [key, v] : ib->map_vertices_info_)
                vs.emplace_back(key, dynamic_cast<const lbmproject::GeometryVertexImmersedBoundary*>(v.get()));
            std::sort(vs.begin(), vs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            std::vector<double> xyz, uvw, area;
            for (const auto& [key, v] : vs) {
                for (int a = 0; a < 3; ++a) {
                    xyz.push_back(a < dims ? v->coordinate_[a] : 0.);
                    uvw.push_back(v->velocity_[a]);
                }
                area.push_back(v->area_);
            }
            Check(zl_ib_set_vertices(ctx_, ib->GetLevel(), static_cast<int64_t>(area.size()), xyz.data(), uvw.data(),
                                     area.data()));
        }
    }
}

void B200Session::StepLevel(DefInt level, DefInt time_step_level) {
    Check(zl_step_level(ctx_, level));
    // InformationFromGridOfDifferentLevel (lbm_solver_interface.cpp:224-238)
    if (level > 0 && time_step_level % 2 == 0) Check(zl_transfer_levels(ctx_, level));
}

void B200Session::Download(const amrproject::GridManagerInterface& gm) const {
    if (!ctx_) return;
    for (std::size_t l = 0; l < codes_.size(); ++l) {
        auto& grid = dynamic_cast<lbmproject::GridInfoLbmInteface&>(*gm.vec_ptr_grid_info_.at(l));
        auto& nodes = *grid.GetPtrToLbmGrid();
        const std::vector<uint64_t>& codes = codes_[l];
        if (codes.empty()) continue;
        const std::size_t q = nodes.begin()->second->f_.size();
        std::vector<double> f(codes.size() * q);
        Check(zl_get_populations(ctx_, static_cast<int>(l), nullptr, f.data(), static_cast<int64_t>(codes.size())));
        for (std::size_t i = 0; i < codes.size(); ++i)
            std::copy_n(&f[i * q], q, nodes.at(DefSFBitset(codes[i]))->f_.begin());
    }
}

void GridInfoLbmB200::AdvancingAtCurrentTime(const amrproject::ETimeSteppingScheme,
                                             const DefInt time_step_level, const DefReal,
                                             amrproject::MpiManager* const,
                                             amrproject::CriterionManager* const ptr_criterion_manager) {
    auto solver = std::dynamic_pointer_cast<lbmproject::SolverLbmInterface>(ptr_solver_.lock());
    if (!solver) amrproject::LogManager::LogError("LBM solver is not created.");
    session_->EnsureUploaded(*GetPtrToParentGridManager(), *solver, ptr_criterion_manager);
    session_->StepLevel(i_level_, time_step_level);
}

}  // namespace zllbm
}  // namespace rootproject
