// GridInfoLbmB200: the reference's LBM grid information (GridInfoLbmInteface,
// lbm_project/lbm_interface.h:201-279) whose per-level time step -- AdvancingAtCurrentTime,
// lbm_project/lbm_grid_interface.cpp:104-153: collide, stream, domain boundaries, immersed-boundary
// forcing, and the coarse/fine exchange of InformationFromGridOfDifferentLevel,
// lbm_solver_interface.cpp:224-238 -- runs on one B200 through the zllbm_b200 C ABI.
//
// Host-side code a ZLLBM maintainer compiles into the reference: it includes the reference's
// headers and links the reference's libraries and libzllbm_b200.so.  Everything else of the
// reference is unchanged: grid generation (AmrManager::SetupMesh), the application's initial
// fields, AmrManager::TimeMarching and its sub-cycled level order, output and checkpoints.
//
//     rootproject::zllbm::B200Session session(options);
//     amr->AddSolverToGridManager(creator);
//     session.Install(solver);                   // before SetSameSolverDependentInfoForAllGrids
//     amr->SetSameSolverDependentInfoForAllGrids(solver_ptr);
//     ... InitializeAllSolvers, SetupMesh, initial fields ...
//     for (it ...) amr->TimeMarching(it);        // the first level step hands the grid over
//     session.Download(*amr->ptr_grid_manager_);  // f_ back into the nodes (output, checkpoint)
//
// The first AdvancingAtCurrentTime hands every level over to the device: node codes and f_,
// interface layers (explosion targets, coalescence targets, coarse-to-fine ghosts) and the
// vertices of immersed-boundary geometries.  Errors go to LogManager::LogError, the reference's
// convention (amr_project/io/log_write.cpp:143-182).
#ifndef ZLLBM_B200_PLUGIN_GRID_INFO_LBM_B200_H_
#define ZLLBM_B200_PLUGIN_GRID_INFO_LBM_B200_H_
#include <map>
#include <memory>
#include <vector>
#include "./lbm_interface.h"
#include "zllbm_b200.h"

namespace rootproject {
namespace zllbm {

struct B200Options {
    int storage = ZL_STORAGE_F64;  // population storage on the device (ZL_STORAGE_*)
    int device = 0;
    // Wall / inflow velocity of each face, as the application passed it to
    // BoundaryConditionLbmInterface::SetValues (the reference keeps it protected).
    std::map<amrproject::EDomainBoundaryDirection, std::vector<DefReal>> boundary_values;
    // Smagorinsky on the device: tau0 + tau_sgs with Cs (the reference's own LES sets
    // tau = tau_sgs, lbm_solver_interface.cpp:291-295, which the library treats as a bug)
    bool les = false;
    DefReal les_cs = 0.16;
};

class B200Session {
 public:
    explicit B200Session(B200Options options) : options_(std::move(options)) {}
    ~B200Session();
    B200Session(const B200Session&) = delete;
    B200Session& operator=(const B200Session&) = delete;

    // The solver creates GridInfoLbmB200 levels from now on (replaces its GridInfoLbmIntefaceCreator).
    void Install(lbmproject::SolverLbmInterface* solver);
    // Hands the grid over once (called by the first level step).
    void EnsureUploaded(const amrproject::GridManagerInterface& grid_manager,
                        const lbmproject::SolverLbmInterface& solver,
                        const amrproject::CriterionManager* criterion_manager);
    // One time step of a level, then the coarse/fine exchange on even sub-steps.
    void StepLevel(DefInt level, DefInt time_step_level);
    // Populations back into GridNodeLbm::f_ of every level.
    void Download(const amrproject::GridManagerInterface& grid_manager) const;

    zl_ctx* context() const { return ctx_; }

 private:
    B200Options options_;
    zl_ctx* ctx_ = nullptr;
    std::vector<std::vector<uint64_t>> codes_;  // per level, the node map's order
    void Check(int rc) const;
};

class GridInfoLbmB200 : public lbmproject::GridInfoLbmInteface {
 public:
    explicit GridInfoLbmB200(B200Session* session) : session_(session) {}
    void AdvancingAtCurrentTime(const amrproject::ETimeSteppingScheme time_scheme,
        const DefInt time_step_level, const DefReal time_step_current,
        amrproject::MpiManager* const ptr_mpi_manager,
        amrproject::CriterionManager* const ptr_criterion_manager) override;

 private:
    B200Session* session_;
};

class GridInfoLbmB200Creator : public amrproject::GridInfoCreatorInterface {
 public:
    explicit GridInfoLbmB200Creator(B200Session* session) : session_(session) {}
    std::shared_ptr<amrproject::GridInfoInterface> CreateGridInfo() const override {
        return std::make_shared<GridInfoLbmB200>(session_);
    }

 private:
    B200Session* session_;
};

}  // namespace zllbm
}  // namespace rootproject
#endif  // ZLLBM_B200_PLUGIN_GRID_INFO_LBM_B200_H_
