// Oracle harness: drives the reference ZLLBM solver through its own public API
// (the same calls examples/lbm/immersed_boundary/cylinder2d/cylinder2d.cpp:14-111
// makes) on a single uniform level, and dumps every node's populations so the
// CUDA path can be compared node by node.  Test infrastructure only.
//
// usage: zl_ref_run key=value ...
//   dims=2|3  n=NX,NY[,NZ] (domain size in cells, dx = 1)  steps=K
//   coll=srt|mrt  nu=<lattice viscosity>  les=0|1
//   bc=<face>:<bb|per|neq>[:ux,uy[,uz]]  (repeatable; faces xmin xmax ymin ymax zmin zmax)
//   init=eq|tgv  u0=<TGV amplitude>  rho0=<default density>  vel=ux,uy[,uz] (initial uniform)
//   out0=<file>  out=<file>  (binary dumps before and after stepping; optional)
//   ckpt=<prefix>  (after stepping, the reference's checkpoint folder <prefix>_checkpoint<step>)
//   rout=<file>  (after stepping: int32 levels, then per level int64 n and n records of uint64 code,
//                 double rho_, sorted by code)
//   vtu=<prefix> vtu_binary=0|1  (after stepping and rout, the reference's own field output
//                 IoManager::OutputMeshData: folder <prefix>_data with per-level .vtu and a .pvtu)
//   timing=1 (print wall-clock seconds of the TimeMarching loop)  warmup=W (untimed steps first)
//   fhist=<file>  (immersed boundary: the vertex force sum after every background step)
//   b200=f64|f32  (only in the zl_ref_run_b200 build: the levels' AdvancingAtCurrentTime runs on the
//                  GPU through the GridInfoLbmB200 plugin, storage f64 or f32; populations are
//                  brought back into the nodes before the dumps)
//
// Dump format (little endian): int32 dims, int32 q, int64 n, then n records of
// uint64 morton code, int32 flag, int32 pad, double f[q]; records sorted by code.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include "./amr_manager.h"
#include "d2q9_model/lbm_d2q9.h"
#include "d3q19_model/lbm_d3q19.h"
#include "criterion/geometry_info_origin.h"
#include "criterion/geometry_default_shape.h"
#include "immersed_boundary/immersed_boundary.h"
#include "immersed_boundary/geometry_ib_shape.h"
#include "les_models/lbm_les_models.h"
#ifdef ZL_B200_PLUGIN
#include "grid_info_lbm_b200.h"
#endif

using namespace rootproject;
using amrproject::EDomainBoundaryDirection;
using lbmproject::ELbmBoundaryConditionScheme;

namespace {
std::vector<double> parse_list(const std::string& s) {
    std::vector<double> v;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ',')) v.push_back(std::atof(tok.c_str()));
    return v;
}

struct FaceBc {
    EDomainBoundaryDirection dir;
    ELbmBoundaryConditionScheme kind;
    std::vector<double> vel;
};

EDomainBoundaryDirection face_of(const std::string& f) {
    if (f == "xmin") return EDomainBoundaryDirection::kBoundaryXMin;
    if (f == "xmax") return EDomainBoundaryDirection::kBoundaryXMax;
    if (f == "ymin") return EDomainBoundaryDirection::kBoundaryYMin;
    if (f == "ymax") return EDomainBoundaryDirection::kBoundaryYMax;
    if (f == "zmin") return EDomainBoundaryDirection::kBoundaryZMin;
    if (f == "zmax") return EDomainBoundaryDirection::kBoundaryZMax;
    std::fprintf(stderr, "unknown face %s\n", f.c_str());
    std::exit(2);
}

ELbmBoundaryConditionScheme kind_of(const std::string& k) {
    if (k == "bb") return ELbmBoundaryConditionScheme::kBounceBack;
    if (k == "per") return ELbmBoundaryConditionScheme::kPeriodic;
    if (k == "neq") return ELbmBoundaryConditionScheme::kNonEqExtrapolation;
    std::fprintf(stderr, "unknown bc kind %s\n", k.c_str());
    std::exit(2);
}

// Multi-level dump: int32 dims, q, nlevels; per level: int64 n, then n records of
// uint64 code, int32 flag, int32 pad, double rho, double u[3], double f[q] (sorted by code);
// then 8 layer lists (inner c2f, outer c2f, inner f2c, outer f2c; each for layers 0..),
// written as int32 kind, int32 layer, int64 count, uint64 codes[count]; terminated by kind -1.
void dump_levels(const std::string& path, int dims, int q, amrproject::GridManagerInterface& gm) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) { std::perror(path.c_str()); std::exit(3); }
    int32_t hdr[3] = {dims, q, static_cast<int32_t>(gm.vec_ptr_grid_info_.size())};
    std::fwrite(hdr, sizeof(hdr), 1, fp);
    for (auto& g : gm.vec_ptr_grid_info_) {
        auto& nodes = *dynamic_cast<lbmproject::GridInfoLbmInteface&>(*g).GetPtrToLbmGrid();
        std::vector<std::pair<uint64_t, lbmproject::GridNodeLbm*>> order;
        for (auto& it : nodes) order.emplace_back(it.first.to_ullong(), it.second.get());
        std::sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        int64_t n = static_cast<int64_t>(order.size());
        std::fwrite(&n, sizeof(n), 1, fp);
        for (auto& [code, node] : order) {
            int32_t fl[2] = {node->flag_status_, 0};
            double mac[4] = {node->rho_, 0., 0., 0.};
            for (size_t a = 0; a < node->velocity_.size() && a < 3; ++a) mac[1 + a] = node->velocity_[a];
            std::fwrite(&code, sizeof(code), 1, fp);
            std::fwrite(fl, sizeof(fl), 1, fp);
            std::fwrite(mac, sizeof(mac), 1, fp);
            std::fwrite(node->f_.data(), sizeof(double), q, fp);
        }
        auto write_layers = [&](int32_t kind, const std::vector<DefMap<DefInt>>& layers) {
            for (size_t i = 0; i < layers.size(); ++i) {
                std::vector<uint64_t> codes;
                for (auto& it : layers[i]) codes.push_back(it.first.to_ullong());
                std::sort(codes.begin(), codes.end());
                int32_t kl[2] = {kind, static_cast<int32_t>(i)};
                int64_t c = static_cast<int64_t>(codes.size());
                std::fwrite(kl, sizeof(kl), 1, fp);
                std::fwrite(&c, sizeof(c), 1, fp);
                std::fwrite(codes.data(), sizeof(uint64_t), codes.size(), fp);
            }
        };
        for (auto& [key, info] : g->map_ptr_interface_layer_info_) {
            write_layers(0, info->vec_inner_coarse2fine_);
            write_layers(1, info->vec_outer_coarse2fine_);
            write_layers(2, info->vec_inner_fine2coarse_);
            write_layers(3, info->vec_outer_fine2coarse_);
        }
        int32_t end[2] = {-1, 0};
        std::fwrite(end, sizeof(end), 1, fp);
    }
    std::fclose(fp);
}

void dump(const std::string& path, int dims, int q, amrproject::GridInfoInterface& grid) {
    auto& nodes = *dynamic_cast<lbmproject::GridInfoLbmInteface&>(grid).GetPtrToLbmGrid();
    std::vector<std::pair<uint64_t, lbmproject::GridNodeLbm*>> order;
    order.reserve(nodes.size());
    for (auto& it : nodes) order.emplace_back(it.first.to_ullong(), it.second.get());
    std::sort(order.begin(), order.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) { std::perror(path.c_str()); std::exit(3); }
    int32_t hdr[2] = {dims, q};
    int64_t n = static_cast<int64_t>(order.size());
    std::fwrite(hdr, sizeof(hdr), 1, fp);
    std::fwrite(&n, sizeof(n), 1, fp);
    for (auto& [code, node] : order) {
        int32_t fl[2] = {node->flag_status_, 0};
        std::fwrite(&code, sizeof(code), 1, fp);
        std::fwrite(fl, sizeof(fl), 1, fp);
        std::fwrite(node->f_.data(), sizeof(double), q, fp);
    }
    std::fclose(fp);
}
}  // namespace

// mode=morton dims=D in=<file of uint64 codes> out=<file>: for every code write the reference's
// FindXNeg, FindXPos, FindYNeg, FindYPos[, FindZNeg, FindZPos] (grid/morton_aux.hpp:65-297).
int morton_mode(int dims, const std::string& in, const std::string& out) {
    FILE* fi = std::fopen(in.c_str(), "rb");
    if (!fi) return 3;
    std::vector<uint64_t> codes;
    uint64_t v;
    while (std::fread(&v, sizeof(v), 1, fi) == 1) codes.push_back(v);
    std::fclose(fi);
    std::vector<uint64_t> res;
    amrproject::SFBitsetAux2D a2;
    amrproject::SFBitsetAux3D a3;
    a2.SFBitsetInitial();
    a3.SFBitsetInitial();
    for (uint64_t c : codes) {
        DefSFBitset b(c);
        if (dims == 2) {
            for (DefSFBitset r : {a2.FindXNeg(b), a2.FindXPos(b), a2.FindYNeg(b), a2.FindYPos(b)})
                res.push_back(r.to_ullong());
        } else {
            for (DefSFBitset r : {a3.FindXNeg(b), a3.FindXPos(b), a3.FindYNeg(b), a3.FindYPos(b),
                                  a3.FindZNeg(b), a3.FindZPos(b)})
                res.push_back(r.to_ullong());
        }
    }
    FILE* fo = std::fopen(out.c_str(), "wb");
    if (!fo) return 3;
    std::fwrite(res.data(), sizeof(uint64_t), res.size(), fo);
    std::fclose(fo);
    return 0;
}

// mode=les dims=D out=<file>: the reference's Smagorinsky increment (LesModelSmagorinsky,
// les_models/lbm_les_smagorinsky.cpp:22-94) on deterministic pseudo-random inputs.  Record:
// double tau0, dt, f[q], feq[q], force[3], u[3], tau_sgs_without_force, tau_sgs_with_force.
int les_mode(int dims, const std::string& out) {
    lbmproject::SolverLbmD2Q9 s2;
    lbmproject::SolverLbmD3Q19 s3;
    lbmproject::SolverLbmInterface& solver = dims == 2 ? static_cast<lbmproject::SolverLbmInterface&>(s2)
                                                       : static_cast<lbmproject::SolverLbmInterface&>(s3);
    const int q = solver.k0NumQ_;
    lbmproject::LesModelSmagorinsky model;
    const lbmproject::LesModelInterface& les = model;
    uint64_t state = 20261203ull;
    auto next = [&state]() {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return static_cast<double>(state >> 11) / 9007199254740992.;
    };
    FILE* fp = std::fopen(out.c_str(), "wb");
    for (int sample = 0; sample < 200; ++sample) {
        lbmproject::GridNodeLbm node;
        node.f_.resize(q);
        node.velocity_.assign(dims, 0.);
        std::vector<double> feq(q), force(3);
        const double tau0 = 0.5 + next();
        const double dt = 1. / static_cast<double>(1 << (sample % 3));
        for (int i = 0; i < q; ++i) {
            feq[i] = solver.k0Weights_[i] * (1. + 0.1 * (next() - 0.5));
            node.f_[i] = feq[i] + 0.01 * (next() - 0.5);
        }
        for (int a = 0; a < 3; ++a) force[a] = 1e-3 * (next() - 0.5);
        for (int a = 0; a < dims; ++a) node.velocity_[a] = 0.1 * (next() - 0.5);
        std::vector<double> fvec(force.begin(), force.begin() + dims);
        const double without = les.CalSgsRelaxationTimeWithoutForce(dt, tau0, feq, node, solver);
        const double with = les.CalSgsRelaxationTimeWithForce(dt, tau0, feq, fvec, node, solver);
        double u3[3] = {node.velocity_[0], node.velocity_[1], dims == 3 ? node.velocity_[2] : 0.};
        std::fwrite(&tau0, 8, 1, fp);
        std::fwrite(&dt, 8, 1, fp);
        std::fwrite(node.f_.data(), 8, q, fp);
        std::fwrite(feq.data(), 8, q, fp);
        std::fwrite(force.data(), 8, 3, fp);
        std::fwrite(u3, 8, 3, fp);
        std::fwrite(&without, 8, 1, fp);
        std::fwrite(&with, 8, 1, fp);
    }
    std::fclose(fp);
    return 0;
}

int main(int argc, char* argv[]) {
    std::map<std::string, std::string> kv;
    std::vector<FaceBc> bcs;
    for (int i = 1; i < argc; ++i) {
        std::string a(argv[i]);
        auto eq = a.find('=');
        if (eq == std::string::npos) continue;
        std::string k = a.substr(0, eq), v = a.substr(eq + 1);
        if (k == "bc") {
            std::stringstream ss(v);
            std::string face, kind, vel;
            std::getline(ss, face, ':');
            std::getline(ss, kind, ':');
            std::getline(ss, vel, ':');
            bcs.push_back({face_of(face), kind_of(kind), vel.empty() ? std::vector<double>{} : parse_list(vel)});
        } else {
            kv[k] = v;
        }
    }
    const int dims = kv.count("dims") ? std::atoi(kv["dims"].c_str()) : 2;
    if (kv.count("mode") && kv["mode"] == "morton") return morton_mode(dims, kv["in"], kv["out"]);
    if (kv.count("mode") && kv["mode"] == "les") return les_mode(dims, kv["out"]);
    const std::vector<double> n = parse_list(kv.count("n") ? kv["n"] : "16,16,16");
    const int steps = kv.count("steps") ? std::atoi(kv["steps"].c_str()) : 1;
    const std::string coll = kv.count("coll") ? kv["coll"] : "srt";
    const double nu = kv.count("nu") ? std::atof(kv["nu"].c_str()) : 0.1;
    const double rho0 = kv.count("rho0") ? std::atof(kv["rho0"].c_str()) : 1.0;
    const std::string init = kv.count("init") ? kv["init"] : "eq";
    const double u0 = kv.count("u0") ? std::atof(kv["u0"].c_str()) : 0.05;
    std::vector<double> vel0 = kv.count("vel") ? parse_list(kv["vel"]) : std::vector<double>(dims, 0.);
    vel0.resize(dims, 0.);

    amrproject::AmrManager* amr = amrproject::AmrManager::GetInstance();
    amr->StartupAmrManager(argc, argv);
    amr->StartupInitialization(dims);
    const int max_level = kv.count("levels") ? std::atoi(kv["levels"].c_str()) : 0;
    amr->ptr_grid_manager_->SetMaxLevel(max_level);
    amr->program_name_ = "zl_ref_run";
    // optional refinement around a default shape (no immersed-boundary forcing):
    //   geo=circle:cx,cy,r  or  geo=cube:cx,cy,cz,edge ; ext=<outer layers per level> ; inner=<layers>
    // immersed-boundary geometry: ib=circle:cx,cy,r (2D) or ib=sphere:cx,cy,cz,r (3D), at level `levels`
    std::shared_ptr<lbmproject::GeometryInfoImmersedBoundary> ib_geo;
    if (kv.count("ib")) {
        const std::string g = kv["ib"];
        const std::string kind = g.substr(0, g.find(':'));
        const std::vector<double> gp = parse_list(g.substr(g.find(':') + 1));
        lbmproject::GeometryInfoImmersedBoundaryCreator creator;
        amr->ptr_criterion_manager_->vec_ptr_geometries_.push_back(creator.CreateGeometryInfo(dims));
        ib_geo = std::dynamic_pointer_cast<lbmproject::GeometryInfoImmersedBoundary>(
            amr->ptr_criterion_manager_->vec_ptr_geometries_.back());
        if (kind == "circle") {
            auto shape = std::make_unique<lbmproject::GeoShapeIBCircle2D>(ib_geo);
            shape->center_ = {gp[0], gp[1]};
            shape->radius_ = gp[2];
            ib_geo->ptr_geo_shape_ = std::move(shape);
        } else {
            auto shape = std::make_unique<lbmproject::GeoShapeIBSphere3D>(ib_geo);
            shape->center_ = {gp[0], gp[1], gp[2]};
            shape->radius_ = gp[3];
            ib_geo->ptr_geo_shape_ = std::move(shape);
        }
        ib_geo->SetGridExtendType(amrproject::EGridExtendType::kInAndOut);
        ib_geo->SetLevel(max_level);
        std::vector<DefInt> ext;
        for (double v : parse_list(kv.count("ext") ? kv["ext"] : "4")) ext.push_back(static_cast<DefInt>(v));
        ext.resize(max_level + 1, ext.back());
        std::vector<DefInt> inner;
        for (double v : parse_list(kv.count("inner") ? kv["inner"] : "4")) inner.push_back(static_cast<DefInt>(v));
        inner.resize(max_level + 1, inner.back());
        ib_geo->SetXExtendPositive(ext);
        ib_geo->SetXExtendNegative(ext);
        ib_geo->SetYExtendPositive(ext);
        ib_geo->SetYExtendNegative(ext);
        if (dims == 3) {
            ib_geo->SetZExtendPositive(ext);
            ib_geo->SetZExtendNegative(ext);
        }
        ib_geo->SetInnerExtend(inner);
        amr->ptr_grid_manager_->vec_ptr_tracking_info_creator_.push_back(
            std::make_unique<amrproject::TrackingGridInfoCreatorInterface>());
        ib_geo->SetPtrTrackingGridInfoCreator(amr->ptr_grid_manager_->vec_ptr_tracking_info_creator_.back().get());
    }
    if (kv.count("geo") && max_level > 0) {
        const std::string g = kv["geo"];
        const std::string kind = g.substr(0, g.find(':'));
        const std::vector<double> gp = parse_list(g.substr(g.find(':') + 1));
        amrproject::GeometryInfoOriginCreator creator;
        amr->ptr_criterion_manager_->vec_ptr_geometries_.push_back(creator.CreateGeometryInfo(dims));
        auto geo = amr->ptr_criterion_manager_->vec_ptr_geometries_.back();
        if (kind == "circle") {
            auto shape = std::make_unique<amrproject::GeoShapeDefaultCircle2D>(geo);
            shape->center_ = {gp[0], gp[1]};
            shape->radius_ = gp[2];
            geo->ptr_geo_shape_ = std::move(shape);
        } else {
            auto shape = std::make_unique<amrproject::GeoShapeDefaultCube3D>(geo);
            shape->center_ = {gp[0], gp[1], gp[2]};
            shape->length_ = gp[3];
            geo->ptr_geo_shape_ = std::move(shape);
        }
        geo->SetGridExtendType(amrproject::EGridExtendType::kInAndOut);
        geo->SetLevel(max_level);
        std::vector<DefInt> ext;
        for (double v : parse_list(kv.count("ext") ? kv["ext"] : "4")) ext.push_back(static_cast<DefInt>(v));
        ext.resize(max_level + 1, ext.back());
        std::vector<DefInt> inner;
        for (double v : parse_list(kv.count("inner") ? kv["inner"] : "4")) inner.push_back(static_cast<DefInt>(v));
        inner.resize(max_level + 1, inner.back());
        geo->SetXExtendPositive(ext);
        geo->SetXExtendNegative(ext);
        geo->SetYExtendPositive(ext);
        geo->SetYExtendNegative(ext);
        if (dims == 3) {
            geo->SetZExtendPositive(ext);
            geo->SetZExtendNegative(ext);
        }
        geo->SetInnerExtend(inner);
        amr->ptr_grid_manager_->vec_ptr_tracking_info_creator_.push_back(
            std::make_unique<amrproject::TrackingGridInfoCreatorInterface>());
        geo->SetPtrTrackingGridInfoCreator(amr->ptr_grid_manager_->vec_ptr_tracking_info_creator_.back().get());
    }
    std::vector<double> domain(n.begin(), n.begin() + dims);
    amr->ptr_grid_manager_->SetDomainSize(domain);
    amr->ptr_grid_manager_->SetDomainGridSize({1.});
    amr->SetupInputDependentParameters();
    lbmproject::SolverCreatorLbmD2Q9 c2;
    lbmproject::SolverCreatorLbmD3Q19 c3;
    if (dims == 2) {
        amr->AddSolverToGridManager(c2);
    } else {
        amr->AddSolverToGridManager(c3);
    }
#ifdef ZL_B200_PLUGIN
    std::unique_ptr<zllbm::B200Session> b200;
    if (kv.count("b200")) {
        zllbm::B200Options opt;
        opt.storage = kv["b200"] == "f32" ? ZL_STORAGE_F32 : ZL_STORAGE_F64;
        for (auto& bc : bcs) {
            std::vector<double> v = bc.vel;
            v.resize(dims, 0.);
            opt.boundary_values[bc.dir] = v;
        }
        b200 = std::make_unique<zllbm::B200Session>(opt);
        b200->Install(dynamic_cast<lbmproject::SolverLbmInterface*>(amr->ptr_grid_manager_->vec_ptr_solver_.at(0).get()));
    }
#endif
    amr->SetSameSolverDependentInfoForAllGrids(amr->ptr_grid_manager_->vec_ptr_solver_.at(0));
    auto& solver = *dynamic_cast<lbmproject::SolverLbmInterface*>(
        amr->ptr_grid_manager_->vec_ptr_solver_.at(0).get());
    for (auto& g : amr->ptr_grid_manager_->vec_ptr_grid_info_) {
        auto& grid = *dynamic_cast<lbmproject::GridInfoLbmInteface*>(g.get());
        solver.SetCollisionOperator(grid.GetGridLevel(), coll == "mrt"
            ? lbmproject::ELbmCollisionOperatorType::kLbmMrt : lbmproject::ELbmCollisionOperatorType::kLbmSrt);
        for (auto& bc : bcs) {
            solver.SetDomainBoundaryCondition(bc.dir, bc.kind, &grid.domain_boundary_condition_);
            std::vector<double> v = bc.vel;
            v.resize(dims, 0.);
            grid.domain_boundary_condition_.at(bc.dir)->SetValues(v);
        }
    }
    if (kv.count("les") && kv["les"] == "1") solver.SetLesModel(lbmproject::ELbmLesModelType::kSmagorinsky);
    if (ib_geo || kv.count("forces")) {
        for (auto& g : amr->ptr_grid_manager_->vec_ptr_grid_info_) (void)g;
        solver.SetNumForces(dims);
    }
    if (kv.count("cforce")) {
        std::vector<double> cf = parse_list(kv["cforce"]);
        cf.resize(dims, 0.);
        solver.SetConstantForce(cf);
    }
    solver.SetDefaultViscosity(nu);
    solver.SetDefaultDensity(rho0);
    solver.SetDefaultVelocity(vel0);
    amr->InitializeAllSolvers();
    amr->SetupMesh(0);

    auto& grid0 = *amr->ptr_grid_manager_->vec_ptr_grid_info_.at(0);
    const int q = solver.k0NumQ_;
    if (init == "tgv") {
        // Taylor-Green vortex written into the public node members after SetupMesh.  The
        // coordinate is taken modulo the period so the duplicated maximum plane of a periodic
        // axis starts bit-identical to the minimum plane.
        auto& nodes = *dynamic_cast<lbmproject::GridInfoLbmInteface&>(grid0).GetPtrToLbmGrid();
        auto* aux3 = dynamic_cast<amrproject::SFBitsetAux3D*>(amr->ptr_grid_manager_.get());
        auto* aux2 = dynamic_cast<amrproject::SFBitsetAux2D*>(amr->ptr_grid_manager_.get());
        const double two_pi = 2. * std::acos(-1.);
        for (auto& it : nodes) {
            double x, y, z = 0.;
            if (dims == 3) {
                std::array<DefAmrLUint, 3> idx;
                aux3->SFBitsetComputeIndices(it.first, &idx);
                x = two_pi * ((idx[0] - 1) % static_cast<DefAmrLUint>(n[0])) / n[0];
                y = two_pi * ((idx[1] - 1) % static_cast<DefAmrLUint>(n[1])) / n[1];
                z = two_pi * ((idx[2] - 1) % static_cast<DefAmrLUint>(n[2])) / n[2];
            } else {
                std::array<DefAmrLUint, 2> idx;
                aux2->SFBitsetComputeIndices(it.first, &idx);
                x = two_pi * ((idx[0] - 1) % static_cast<DefAmrLUint>(n[0])) / n[0];
                y = two_pi * ((idx[1] - 1) % static_cast<DefAmrLUint>(n[1])) / n[1];
            }
            std::vector<double> u(dims);
            u[0] = u0 * std::sin(x) * std::cos(y) * std::cos(z);
            u[1] = -u0 * std::cos(x) * std::sin(y) * std::cos(z);
            if (dims == 3) u[2] = 0.;
            const double p = (dims == 3)
                ? rho0 * u0 * u0 / 16. * (std::cos(2. * x) + std::cos(2. * y)) * (std::cos(2. * z) + 2.)
                : rho0 * u0 * u0 / 4. * (std::cos(2. * x) + std::cos(2. * y));
            const double rho = rho0 + 3. * p;
            solver.func_cal_feq_(rho, u, &it.second->f_);
            it.second->f_collide_ = it.second->f_;
            it.second->rho_ = rho;
            it.second->velocity_ = u;
        }
    }
    auto dump_vertices = [&](const std::string& path) {
        // int64 n, then per vertex (sorted by key): double coord[3], vel[3], area, force[3]
        FILE* fp = std::fopen(path.c_str(), "wb");
        std::vector<std::pair<DefSizet, lbmproject::GeometryVertexImmersedBoundary*>> vs;
        for (auto& [key, v] : ib_geo->map_vertices_info_)
            vs.emplace_back(key, dynamic_cast<lbmproject::GeometryVertexImmersedBoundary*>(v.get()));
        std::sort(vs.begin(), vs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        int64_t n = static_cast<int64_t>(vs.size());
        std::fwrite(&n, sizeof(n), 1, fp);
        for (auto& [key, v] : vs) {
            double rec[10] = {v->coordinate_[0], v->coordinate_[1], dims == 3 ? v->coordinate_[2] : 0.,
                              v->velocity_[0], v->velocity_[1], v->velocity_[2], v->area_,
                              v->force_[0], v->force_[1], v->force_[2]};
            std::fwrite(rec, sizeof(rec), 1, fp);
        }
        std::fclose(fp);
    };
    if (ib_geo && kv.count("vout0")) dump_vertices(kv["vout0"]);
    if (kv.count("lout0")) dump_levels(kv["lout0"], dims, q, *amr->ptr_grid_manager_);
    if (kv.count("out0")) dump(kv["out0"], dims, q, grid0);
    const int warmup = kv.count("warmup") ? std::atoi(kv["warmup"].c_str()) : 0;
    for (int it = 0; it < warmup; ++it) amr->TimeMarching(it);
    auto t0 = std::chrono::steady_clock::now();
    // fhist=<file>: after every background step, the immersed-boundary force sum over the vertices
    // (vertex order by key), sum F area (WriteTimeHisLagrangianForce, immersed_boundary.cpp:596-642,
    // with dx = 1 at the background level): int64 steps, then steps x double[3]
    std::vector<double> fhist;
    for (int it = warmup; it < warmup + steps; ++it) {
        amr->TimeMarching(it);
        if (ib_geo && kv.count("fhist")) {
            std::vector<std::pair<DefSizet, lbmproject::GeometryVertexImmersedBoundary*>> vs;
            for (auto& [key, v] : ib_geo->map_vertices_info_)
                vs.emplace_back(key, dynamic_cast<lbmproject::GeometryVertexImmersedBoundary*>(v.get()));
            std::sort(vs.begin(), vs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            double tot[3] = {0., 0., 0.};
            for (auto& [key, v] : vs)
                for (int d = 0; d < dims; ++d) tot[d] += v->force_[d] * v->area_;
            fhist.insert(fhist.end(), tot, tot + 3);
        }
    }
    auto t1 = std::chrono::steady_clock::now();
#ifdef ZL_B200_PLUGIN
    if (b200) b200->Download(*amr->ptr_grid_manager_);
#endif
    if (kv.count("fhist")) {
        FILE* fp = std::fopen(kv["fhist"].c_str(), "wb");
        if (!fp) { std::perror(kv["fhist"].c_str()); return 3; }
        int64_t nh = static_cast<int64_t>(fhist.size() / 3);
        std::fwrite(&nh, sizeof(nh), 1, fp);
        std::fwrite(fhist.data(), sizeof(double), fhist.size(), fp);
        std::fclose(fp);
    }
    if (kv.count("out")) dump(kv["out"], dims, q, grid0);
    if (kv.count("lout")) dump_levels(kv["lout"], dims, q, *amr->ptr_grid_manager_);
    if (ib_geo && kv.count("vout")) dump_vertices(kv["vout"]);
    if (kv.count("ckpt")) {
        // the reference's own checkpoint writer (IoManager::WriteCheckPointData,
        // io_checkpoint.cpp:27-51): folder <ckpt>_checkpoint<steps> with loadings, grid_nodes,
        // interface_nodes
        const auto t = static_cast<DefAmrLUint>(warmup + steps);
        if (dims == 2) {
            auto& gm = dynamic_cast<amrproject::GridManager2D&>(*amr->ptr_grid_manager_);
            amr->ptr_io_manager_->WriteCheckPointData(t, kv["ckpt"], gm, gm, *amr->ptr_criterion_manager_,
                                                      *amr->ptr_mpi_manager_);
        } else {
            auto& gm = dynamic_cast<amrproject::GridManager3D&>(*amr->ptr_grid_manager_);
            amr->ptr_io_manager_->WriteCheckPointData(t, kv["ckpt"], gm, gm, *amr->ptr_criterion_manager_,
                                                      *amr->ptr_mpi_manager_);
        }
    }
    if (kv.count("rout")) {
        // the node member rho_ the reference's "rho" output variable writes (set by the last collision)
        FILE* fp = std::fopen(kv["rout"].c_str(), "wb");
        if (!fp) { std::perror(kv["rout"].c_str()); return 3; }
        auto& infos = amr->ptr_grid_manager_->vec_ptr_grid_info_;
        int32_t nl = static_cast<int32_t>(infos.size());
        std::fwrite(&nl, sizeof(nl), 1, fp);
        for (auto& info : infos) {
            auto& nodes = *dynamic_cast<lbmproject::GridInfoLbmInteface&>(*info).GetPtrToLbmGrid();
            std::vector<std::pair<uint64_t, double>> rr;
            for (auto& it : nodes) rr.emplace_back(it.first.to_ullong(), it.second->rho_);
            std::sort(rr.begin(), rr.end());
            int64_t nr = static_cast<int64_t>(rr.size());
            std::fwrite(&nr, sizeof(nr), 1, fp);
            for (auto& [code, rho] : rr) {
                std::fwrite(&code, sizeof(code), 1, fp);
                std::fwrite(&rho, sizeof(rho), 1, fp);
            }
        }
        std::fclose(fp);
    }
    if (kv.count("vtu")) {
        auto& io = *amr->ptr_io_manager_;
        io.bool_binary_ = !kv.count("vtu_binary") || std::atoi(kv["vtu_binary"].c_str()) != 0;
        io.SetupOutputFormat();
        io.SetupDependentIOParameters();
        io.OutputMeshData(kv["vtu"], amr->ptr_grid_manager_.get(), amr->ptr_criterion_manager_.get());
    }
    if (kv.count("timing")) {
        const double sec = std::chrono::duration<double>(t1 - t0).count();
        std::printf("{\"nodes\": %zu, \"steps\": %d, \"seconds\": %.6f}\n", grid0.map_grid_node_.size(), steps, sec);
    }
    return 0;
}
