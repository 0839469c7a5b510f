/*
 * zllbm_b200 — C ABI of the B200 lattice-Boltzmann time step.
 *
 * The library replaces, for one GPU, the per-level time step of the
 * reference ZLLBM LBM plugin: GridInfoLbmInteface::AdvancingAtCurrentTime
 * (lbm_project/lbm_grid_interface.cpp:104-153), which collides every node,
 * pull-streams it through Morton-code hash lookups, applies the domain
 * boundary conditions and exchanges coarse/fine information.  A host
 * (the reference's AmrManager / GridManager, or any other caller) keeps
 * owning the Morton-coded node sets; it hands each level's codes over once,
 * then calls zl_step_level (or zl_advance) where the reference called
 * AdvancingAtCurrentTime.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Arrays passed in are copied; the caller
 *    keeps ownership.  Pointers are HOST pointers unless a name says _device.
 *  - Populations use the reference's direction order (d2q9_model/lbm_d2q9.h:53-61,
 *    d3q19_model/lbm_d3q19.h:18-85) and are exchanged in the order of the
 *    Morton codes the caller passes, q fastest (node-major, like GridNodeLbm::f_).
 *  - Every call returns 0 on success or a negative ZL_E* code; zl_last_error
 *    gives the message.  This replaces the reference's LogError + MPI_Abort
 *    (amr_project/io/log_write.cpp:143-182): a C++ wrapper maps a non-zero
 *    return to LogManager::LogError to keep the reference's behaviour.
 *  - One host thread per context; all work is ordered on the context's own
 *    CUDA stream.  No global mutable state is shared between contexts.
 */
#ifndef ZLLBM_B200_H_
#define ZLLBM_B200_H_
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZL_ABI_VERSION 2
#define ZL_MAX_LEVELS 8

/* error codes */
#define ZL_OK 0
#define ZL_EINVAL (-1)     /* bad argument */
#define ZL_ETOPOLOGY (-2)  /* node codes inconsistent with the level / domain */
#define ZL_EDEVICE (-3)    /* CUDA error */
#define ZL_ETIMEOUT (-4)   /* a bounded device wait gave up */
#define ZL_ENAN (-5)       /* non-finite populations detected */
#define ZL_ESTATE (-6)     /* call out of order (e.g. stepping a level with no nodes) */
#define ZL_ETOOLARGE (-7)  /* input larger than a fixed-capacity entry point accepts */

/* lattice (SolverCreatorLbmD2Q9 / SolverCreatorLbmD3Q19, lbm_d2q9_mandatory.cpp:19-23,
   lbm_d3q19_mandatory.cpp:20-24) */
#define ZL_D2Q9 2
#define ZL_D3Q19 3

/* collision operators (ELbmCollisionOperatorType, collision_model/lbm_collision_models.h:21-25) */
#define ZL_SRT 0
#define ZL_MRT 1

/* domain boundary conditions (ELbmBoundaryConditionScheme,
   boundary_conditions/lbm_boundary_conditions.h:22-27) */
#define ZL_BC_NONE 0
#define ZL_BC_BOUNCE_BACK 1
#define ZL_BC_PERIODIC 2
#define ZL_BC_NONEQ_EXTRAPOLATION 3
/* No counterpart in the reference: populations entering across the face are advected out of the
   inner node, f(x_b) = (f_old(x_b) + U f(x_b - n)) / (1 + U), with U = |bc_velocity[face][axis]| > 0. */
#define ZL_BC_CONVECTIVE_OUTFLOW 4

/* face slots (EDomainBoundaryDirection, amr_project/grid/grid_enumerates.h) */
#define ZL_FACE_XMIN 0
#define ZL_FACE_XMAX 1
#define ZL_FACE_YMIN 2
#define ZL_FACE_YMAX 3
#define ZL_FACE_ZMIN 4
#define ZL_FACE_ZMAX 5

/* rounding of FP16 / BF16 populations written by the step kernels (zl_config.storage_rounding);
   stochastic rounding is the default: round to nearest repeats nearly the same error pattern every
   step on a slowly changing flow and lets it accumulate (TGV 256^3, 5,000 steps: FP16 velocity
   error 1.4e-3 nearest, 3.0e-4 stochastic; BF16 8.0e-2 and 2.4e-3) */
#define ZL_ROUND_STOCHASTIC 0
#define ZL_ROUND_NEAREST 1

/* population storage in device memory */
#define ZL_STORAGE_F64 0  /* raw f in FP64, reference arithmetic order: bit-exact parity mode */
#define ZL_STORAGE_F32 1  /* f - w in FP32, FP32 collision */
#define ZL_STORAGE_F16 2  /* (f - w) * scale in FP16, FP32 collision */
#define ZL_STORAGE_BF16 3 /* (f - w) * scale in BF16, FP32 collision */

/* Solver and domain settings: the values a reference application sets through
   SolverLbmInterface::SetCollisionOperator / SetDomainBoundaryCondition + SetValues /
   SetDefaultViscosity / SetDefaultDensity (lbm_project/lbm_interface.h:298-319,452-465)
   and GridManagerInterface::SetDomainSize / SetMaxLevel (amr_project/grid/grid_manager.h:117-129). */
typedef struct zl_config {
    int lattice;               /* ZL_D2Q9 or ZL_D3Q19 */
    int collision;             /* ZL_SRT or ZL_MRT */
    int storage;               /* ZL_STORAGE_* */
    int max_level;             /* finest refinement level, < ZL_MAX_LEVELS */
    double viscosity;          /* lattice viscosity at the background level (tau_l = 3 nu 2^l + 0.5) */
    double rho0;               /* default density */
    int bc_kind[6];            /* ZL_BC_* per face slot */
    double bc_velocity[6][3];  /* wall / boundary velocity per face slot */
    int32_t domain_min[3];     /* background index range of the domain (the reference starts at 1) */
    int32_t domain_max[3];
    double init_velocity[3];   /* default velocity: nodes start at feq(rho0, init_velocity)
                                  (SetDefaultVelocity, lbm_interface.h:300) */
    double storage_scale;      /* scale of FP16/BF16 deviations (0 selects the default 2^13) */
    int forcing;               /* 1: collide with Guo forcing and per-node forces (SetNumForces /
                                  SetConstantForce, lbm_interface.h:298-319); needed by immersed boundaries.
                                  FP64 storage collides every node with the forcing terms, as the
                                  reference does; FP32/FP16/BF16 levels whose forces are all zero (no
                                  constant force, no vertex set so far) take the unforced update */
    double constant_force[3];  /* SetConstantForce */
    int les;                   /* ZL_LES_SMAGORINSKY: tau = tau0 + tau_sgs (the reference sets tau = tau_sgs,
                                  lbm_solver_interface.cpp:291-295, which this library treats as a bug);
                                  ZL_LES_LEARNED: the same increment with a per-node constant from the
                                  closure network (zl_set_closure), Smagorinsky when none is set */
    double les_cs;             /* Smagorinsky constant (0 selects the reference's 0.16, lbm_les_models.h:49) */
    double dx;                 /* background grid spacing (SetDomainGridSize); 0 selects 1 */
    int device;                /* CUDA device ordinal */
    int storage_rounding;      /* FP16/BF16 storage: ZL_ROUND_STOCHASTIC (default: the step kernels
                                  round each stored population up or down at random, with probability
                                  given by its distance to the two neighbours, from counter-based random
                                  bits; unbiased, deterministic for a given sequence of calls) or
                                  ZL_ROUND_NEAREST.  Uploads, face passes and level transfers round to
                                  nearest. */
} zl_config;

typedef struct zl_ctx zl_ctx;

/* Create a context on config->device.  Replaces SolverCreatorLbm*::CreateSolver plus
   SolverLbmInterface::SolverInitial (lbm_solver_interface.cpp:19-44). */
int zl_create(const zl_config* config, zl_ctx** out);

/* Release every device allocation of the context. */
int zl_destroy(zl_ctx* ctx);

/* Hand over the node set of one refinement level: the Morton codes of
   GridInfoInterface::map_grid_node_ (amr_project/grid/grid_info_interface.h:258), in any
   order.  Codes are decoded and the level's dense device box, presence mask and per-node
   boundary / missing-neighbour flags are built on the device.  Populations start at
   feq(rho0, 0), as GridInfoLbmInteface::InitialGridInfo does (lbm_grid_interface.cpp:176-191). */
int zl_set_level_nodes(zl_ctx* ctx, int level, const uint64_t* codes, int64_t n);

/* Write / read the post-stream populations f_ (GridNodeLbm::f_, lbm_interface.h:37) of the
   nodes with the given codes; f holds n * q doubles, node-major.  On periodic axes the
   reference stores the maximum plane as a duplicate of the minimum plane
   (grid/grid_manager3d.cpp:106-112); both codes address the same device node, which is stored
   once.  zl_set_populations writes that node from the minimum-plane code only and ignores the
   maximum-plane row (the reference keeps the two copies equal; if a caller's copies disagree,
   the minimum-plane copy is kept); zl_get_populations returns the node's values for both codes.
   codes may be NULL: the exchange then covers the level's own node list, in the order given to
   zl_set_level_nodes (n must be its length), which the context keeps on the device, so repeated
   exchanges send no codes.  The device staging of these calls (and of zl_get_macros) grows to the
   largest exchange and stays with the context until zl_destroy, so repeated exchanges allocate
   nothing. */
int zl_set_populations(zl_ctx* ctx, int level, const uint64_t* codes, const double* f, int64_t n);
int zl_get_populations(zl_ctx* ctx, int level, const uint64_t* codes, double* f, int64_t n);

/* Density and velocity recomputed from f_ like the reference's output variables
   (lbm_grid_interface.cpp:614-657): rho[n], u[n * dims]. */
int zl_get_macros(zl_ctx* ctx, int level, const uint64_t* codes, double* rho, double* u, int64_t n);

/* One time step of one level: collide, stream, domain boundary conditions.
   Replaces GridInfoLbmInteface::AdvancingAtCurrentTime (lbm_grid_interface.cpp:104-153)
   for a level without coarse/fine neighbours. */
int zl_step_level(zl_ctx* ctx, int level);

/* Part of a time step of a D3Q19 level: the node updates of planes [first, first + count) of its
   last axis, with the level's current step parity; finish != 0 then completes the step (the next
   call steps the other parity).  Every plane once per step, in any split and order, gives the
   whole step's result bit for bit (the single-buffer AA update of a node touches only its own
   slot set).  A sharded slab steps its interior planes while its halo planes are in flight and its
   boundary planes after they arrive.  For levels without ordered face passes, immersed boundary or
   learned closure; no reference counterpart (the reference updates a level in one pass). */
int zl_step_level_planes(zl_ctx* ctx, int level, int first, int count, int finish);

/* Coarse/fine interface of refinement level `level` (>= 1) with level - 1, from the reference's
   interface layer maps (InterfaceLayerInfo, amr_project/grid/grid_info_interface.h:117-127):
     c2f_fine        fine nodes of the fine-to-coarse layers 1..2 of `level` (vec_{inner,outer}_
                     fine2coarse_), the targets of the explosion (TransferInfoFromCoarseGrid,
                     lbm_grid_interface.cpp:408-515);
     f2c_coarse      coarse nodes of coarse-to-fine layer 1 of `level - 1` (vec_{inner,outer}_
                     coarse2fine_), the targets of the coalescence (TransferInfoToCoarseGrid, :524-564);
     coarse_excluded coarse nodes flagged kNodeStatusCoarse2FineGhost_ (amr_project/grid/grid_manager.h:64-73),
                     which the interpolation skips in favour of the coincident fine node.
   Interpolation stencils (4-point Lagrange per axis, grid/grid_interpolation.cpp:433-525) are
   resolved here; stencils that reach the domain boundary return ZL_ETOPOLOGY. */
int zl_set_level_interface(zl_ctx* ctx, int level, const uint64_t* c2f_fine, int64_t n_c2f,
                           const uint64_t* f2c_coarse, int64_t n_f2c, const uint64_t* coarse_excluded,
                           int64_t n_excluded);

/* Exchange between `fine_level` and fine_level - 1 (SolverLbmInterface::InformationFromGridOfDifferentLevel,
   lbm_solver_interface.cpp:224-238): explosion into the fine ghost layers, then coalescence. */
int zl_transfer_levels(zl_ctx* ctx, int fine_level);

/* n background steps of every level, in the reference's sub-cycled order
   (AmrManager::TimeMarching, amr_manager.cpp:279-300; MultiTimeSteppingC2F,
   grid/grid_manager.cpp:997-1023), with the coarse/fine exchange after every second
   sub-step of a fine level. */
int zl_advance(zl_ctx* ctx, int steps);

/* Time interpolation at coarse/fine interfaces (no counterpart in the reference, whose
   explosion is spatial only and leaves the fine ghost layers stale during odd fine sub-steps,
   lbm_solver_interface.cpp:224-238).  zl_interpolate_interface sets the explosion targets of
   fine_level to 0.5 (their values at the last zl_transfer_levels + the values the coarse
   level's current state gives); with zl_set_temporal_interpolation(ctx, 1), zl_advance does
   that before the second fine sub-step of every pair.  Off by default. */
int zl_set_temporal_interpolation(zl_ctx* ctx, int enabled);
int zl_interpolate_interface(zl_ctx* ctx, int fine_level);

/* In zl_advance, run consecutive level steps that no transfer separates (e.g. levels 0, 1, 2 at
   the start of a sub-cycled step) as one launch of the multi-level kernel.  On by default; the
   results are identical either way (those steps touch disjoint data). */
int zl_set_batching(zl_ctx* ctx, int enabled);

/* In zl_advance of a multi-level context, issue each level's steps, immersed-boundary passes,
   face passes and transfers on a stream of that level (finer levels at higher stream priority),
   each operation waiting only for the last operations on the levels it touches: the background
   level's step overlaps the finer levels' sub-steps and transfers.  On by default, and then
   zl_set_batching has no effect on zl_advance; results are identical either way.  The caller's
   stream (zl_set_stream) waits for all of it before zl_advance returns its work.  No reference
   counterpart (the reference advances the levels one after another,
   amr_project/grid/grid_manager.cpp:997-1023). */
int zl_set_level_streams(zl_ctx* ctx, int enabled);

/* Replay zl_advance as a captured CUDA graph of two background steps (every launch of the
   sub-cycled order, transfers and boundary passes included).  The graph is re-captured after any
   change of levels, interfaces, vertices or tuning.  Off by default. */
int zl_set_graph(zl_ctx* ctx, int enabled);

/* Thread-block shape of a level's step kernel: x (a multiple of 32) by y threads, at most 256;
   a negative x selects the kernel that updates two nodes per thread with packed FP32 pairs
   (full periodic D3Q19 boxes in FP32/FP16/BF16 storage, no forcing or LES); x = ZL_BLOCK_ROW
   selects the kernel that gives each warp one whole x-row (y = 1, 2 or 4 rows per block; full
   periodic D3Q19 boxes in FP16/BF16 storage whose rows hold 128 or 256 nodes, no forcing or
   LES). */
#define ZL_BLOCK_ROW (1 << 20)
int zl_set_block(zl_ctx* ctx, int level, int x, int y);

/* Choose the thread-block shape of a level's step kernel by timing candidate shapes (on a saved
   copy of the populations, which are restored).  chosen[2] (may be NULL) receives {x, y}. */
int zl_autotune(zl_ctx* ctx, int level, int trials, int32_t* chosen);

/* Sum over a level's nodes of rho and rho*u, accumulated in FP64 on the device:
   out[0] = mass, out[1..dims] = momentum.  Non-finite sums return ZL_ENAN. */
int zl_conservation(zl_ctx* ctx, int level, double* out);

/* Wait for all work of the context. */
int zl_synchronize(zl_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order work around it. */
int zl_get_stream(const zl_ctx* ctx, void** stream);

/* Make the context issue its work on a caller-owned cudaStream_t (NULL restores its own stream).
   The caller keeps the stream alive while the context uses it. */
int zl_set_stream(zl_ctx* ctx, void* stream);

/* Copy the last error message (NUL-terminated, truncated to n bytes). */
int zl_last_error(const zl_ctx* ctx, char* buf, size_t n);

/* Number of nodes, box extents (x, y, z) and bytes of population storage of a level. */
int zl_level_info(const zl_ctx* ctx, int level, int64_t* nodes, int32_t* extent, int64_t* pop_bytes);

/* ---- topology helpers (device Morton arithmetic, bit-exact with the reference) ---- */

/* For each code, the six (2D: four) axis neighbours computed on the device with the
   reference's FindXNeg/FindXPos/... (amr_project/grid/morton_aux.hpp:65-297), including
   its rule that a Neg step at a zero axis field returns the input code.  out holds
   n * 2 * dims codes ordered xneg, xpos, yneg, ypos[, zneg, zpos]. */
int zl_morton_neighbors(int dims, const uint64_t* codes, int64_t n, uint64_t* out);

/* For each node i of a code set and each direction q, the position in `codes` of the
   upstream node x - c_q the reference's stream pulls from
   (d3q19_model/lbm_d3q19_solver.cpp:20-136, d2q9_model/lbm_d2q9_solver.cpp:21-82), or -1
   when it is not in the set (the reference then keeps the stale value).  Resolved on the
   device by Morton neighbour arithmetic and binary search; out holds n * q int64. */
int zl_upstream_index(int lattice, const uint64_t* codes, int64_t n, int64_t* out);

/* The MRT collision matrix M^-1 S M for relaxation time tau, built in the reference's loop
   order (collision_model/lbm_collision_model_mrt.cpp:63-82); out holds q * q doubles. */
int zl_mrt_matrix(int lattice, double tau, double* out);

/* ---- immersed boundary (FsiImmersedBoundary, lbm_project/immersed_boundary/immersed_boundary.cpp) ---- */

/* Lagrangian vertices of the immersed-boundary geometries of a level (config->forcing must be 1):
   coordinates and velocities as the reference's GeometryVertexImmersedBoundary coordinate_ /
   velocity_ (n * 3 doubles, domain offset included), area_ (n doubles).  Every later step of the
   level starts with the direct-forcing pass (CalculateBodyForce, :35-364, delta kernel of
   stencil half-width 2, StencilDisTwo :372-384).  Calling it again between steps replaces the
   set (the reference's per-step UpdateShape of a moving geometry, or a body with prescribed
   motion): nodes that only the previous set's stencils touched drop their force, n = 0 removes
   the boundary, and a captured graph is rebuilt on the next zl_advance. */
int zl_ib_set_vertices(zl_ctx* ctx, int level, int64_t n, const double* coordinates, const double* velocity,
                       const double* area);

/* Delta kernel of a level's immersed boundary: ZL_IB_DELTA_4, the reference's four-point
   StencilDisTwo (immersed_boundary.cpp:365-384, the default), or ZL_IB_DELTA_3, the three-point
   kernel of Roma, Peskin and Berger (1999), which the reference does not have.  Set it before
   zl_ib_set_vertices (the stencil check and the list of stencil nodes use it); changing it while
   the level has vertices returns ZL_ESTATE. */
#define ZL_IB_DELTA_4 4
#define ZL_IB_DELTA_3 3
int zl_ib_set_delta(zl_ctx* ctx, int level, int width);

/* Vertex forces of the last forcing pass (n * 3, may be NULL) and their sum F area / dx^(d-1)
   in FP64 (total[3], may be NULL; WriteTimeHisLagrangianForce, :596-642). */
int zl_ib_get_forces(zl_ctx* ctx, int level, double* vertex_forces, double* total);

/* ---------------------------------------------------------------- halo faces (slab sharding)
   A level can be one slab of a lattice split across several contexts (one per GPU), the way the
   reference splits its grid over MPI ranks (halo of one node layer per level sub-step,
   amr_project/mpi/mpi_grid_communication.cpp:210-357).  A halo face has ZL_BC_NONE and the level
   box on the domain face; zl_set_level_halo makes its ghost cells hold the neighbour's slots
   (present for the lookups of the nodes next to them, never stepped).  Single-level contexts
   without forcing.  With the single-buffer AA pattern an even step touches only a node's own
   slots, so a pair of steps needs two exchanges per face:
     stage 0, after an even step: zl_halo_pack(face, 0) on this context -> zl_halo_unpack(opposite
       face, 0) on the neighbour (the boundary plane's populations that enter the neighbour);
     stage 1, after an odd step: zl_halo_pack(face, 1) -> zl_halo_unpack(opposite face, 1) on the
       neighbour (the populations this context's nodes wrote into its ghost plane, which belong to
       the neighbour's boundary nodes).
   Buffers are device buffers of zl_halo_bytes; the populations are the storage's raw elements. */
int zl_set_level_halo(zl_ctx* ctx, int level, int faces); /* faces: bit f = face slot f */
int zl_halo_bytes(zl_ctx* ctx, int level, int face, int64_t* bytes);
int zl_halo_pack(zl_ctx* ctx, int level, int face, int stage, void* buf_device);
int zl_halo_unpack(zl_ctx* ctx, int level, int face, int stage, const void* buf_device);

/* ABI version of the loaded library. */
int zl_abi_version(void);

/* ---- allocation-free entry point (no counterpart in the reference) ---- */

/* Mass and momentum of n nodes, summed in FP64 like zl_conservation, for callers that cannot
   call cudaMalloc (work issued from a loop where cudaMalloc / cudaFree would synchronize the
   device, or device memory owned entirely by another allocator).  It allocates nothing:
     - f_device: caller-owned device array of n * q doubles, node-major (GridNodeLbm::f_ order);
     - out_device: caller-owned device array of 4 doubles {mass, jx, jy, jz} (jz = 0 in 2D);
     - stream: cudaStream_t to issue on (NULL: the legacy default stream).
   Block partial sums go to a fixed static device array of 128 KiB that every GPU loading the
   library keeps until process exit; its capacity caps n at 16,777,216 nodes per call (larger
   n returns ZL_ETOOLARGE).  The first call on a device looks up that array's device address
   with that device current, so make the first call before any stream capture.  The array is
   shared by all calls and keeps the last call's partials; every call rewrites the partials it
   reads, but calls that overlap on the GPU (different streams, or host threads without
   ordering) race on it.  The call is asynchronous on `stream`; read out_device after
   synchronizing. */
int zl_moments_noalloc(int lattice, const double* f_device, int64_t n, double* out_device, void* stream);

/* ---------------------------------------------------------------- checkpoint node records
   The file grid_nodes of the reference's checkpoint folder (MpiManager::WriteCheckPointGridNodes,
   mpi_checkpoint.cpp:272-380; node data GridNodeLbm::CopyANodeToBufferForCheckpoint,
   lbm_interface.h:57-78), from and into the device state, so that runs restart across the
   reference and this library.  Layout: uint32 node count, int32 node data size, then per node
   uint64 code, int32 level, int32 flag, double f[q], double force[dims] (forcing contexts: the
   node forces of the last forcing pass), ordered by background cell (ascending code >> dims *
   level), then level, then x-y-z order inside the cell.  The other files of the folder
   (loadings, interface_nodes) describe the host's grid and stay with the host. */

/* codes[l], flags[l] (the reference's flag_status_, kept by the host) and n[l] list level l's
   nodes, for every level 0 .. max_level. */
int zl_write_checkpoint_nodes(zl_ctx* ctx, const char* path, const uint64_t* const* codes,
                              const int32_t* const* flags, const int64_t* n);
/* Populations of every record into its level (each level's node set must contain the codes);
   flags and forces are left to the host (forces are recomputed by the next forcing pass). */
int zl_read_checkpoint_nodes(zl_ctx* ctx, const char* path);

/* ---------------------------------------------------------------- field output (VTK XML)
   Replaces VtkWriterManager::WriteVtuAll with its default kPartitionMultiBlock option
   (amr_project/io/vtk_writer_manager.cpp:103-190, reached through IoManager::OutputMeshData,
   io/io_manager.cpp:100-112): <prefix>_data/rank_0_grid_level_<l>.vtu for every level and
   <prefix>_data/rank_0_.pvtu listing them, in the reference's layout and number formats
   (binary: base64 of a UInt32 byte count and the data; ascii: the printf formats of
   IoManager::SetupOutputFormat).  Point arrays flag_status (UInt16), vtkGhostType (UInt8: 1 where
   flag & ghost_mask), rho and velocity (Float32, recomputed from the current populations, with
   the node forces on forced levels), coordinates (Float32: origin + spacing / 2^l per set
   Morton bit, SFBitsetComputeCoordinate); VTK_PIXEL / VTK_VOXEL cells for every point whose
   +x/+y/+z corners are all points of the level (SFBitsetBelongToOneCell).  The per-point arrays,
   the cell connectivity and the base64 text are built on the device.
   codes[l], flags[l], n[l]: level l's points in output order (the reference writes its hash-map
   order) with their flag_status; space / origin: the background grid spacing and the coordinate
   of index 0 per axis (-spacing * k0MinIndexOfBackgroundNode_ for the reference's grids).
   The reference writes "rho" before "velocity" recomputes the node macros, so its rho is the node
   member left by the last collision; here rho is the density of the current populations. */
#define ZL_VTU_GHOST_DEFAULT 0x3Eu /* C2F0 | C2F ghost | F2C0 | F2C ghost | MPI outer (NodeBitStatus) */
int zl_write_vtu(zl_ctx* ctx, const char* prefix, int binary, const double* space, const double* origin,
                 uint32_t ghost_mask, const uint64_t* const* codes, const int32_t* const* flags, const int64_t* n);

/* ---------------------------------------------------------------- full-box levels, device I/O
   No counterpart in the reference, whose levels are always hash maps of nodes; these let a
   periodic box of 10^9 nodes be set up and read without host node lists. */

/* Make `level` the full box of n[0] x n[1] x n[2] nodes starting at level index lo (like
   zl_set_level_nodes given every code of the box).  On a periodic axis a box spanning the whole
   domain (n = (domain_max - domain_min) << level) wraps around and stores each plane once. */
int zl_set_level_box(zl_ctx* ctx, int level, const int32_t lo[3], const int32_t n[3]);

/* Set every node of a full-box level to feq(rho, u), from device arrays in box order (x fastest):
   rho_device[n], u_device[n * 3] (FP32); any storage (FP64: feq in the reference's arithmetic). */
int zl_set_equilibrium_dense(zl_ctx* ctx, int level, const float* rho_device, const float* u_device);

/* Density and velocity of every node of a full-box level into device arrays (box order, FP32);
   any storage. */
int zl_get_macros_dense(zl_ctx* ctx, int level, float* rho_device, float* u_device);

/* ---------------------------------------------------------------- learned LES closure
   No counterpart in the reference (it hard-wires Smagorinsky, lbm_les_smagorinsky.cpp:22-94).
   A per-node network y = MLP(x) with x the 24 node features (the 19 non-equilibrium MRT moments
   / rho, tr S, S:S, tr(Sd^3), |Sd| and the Cs = 0.1 Smagorinsky increment, S = -3 Pi / (2 rho tau0))
   gives the Smagorinsky constant C = 18 c with c = 0.01 * clamp(y, 0, 8):
       tau = tau0 + 0.5 * (sqrt(tau0^2 + C sqrt(2 Pi:Pi)) - tau0).
   Network: 24 -> 64 -> 64 -> 1, tanh-form GELU, BF16 tensor-core operands, FP32 accumulation. */
#define ZL_LES_OFF 0
#define ZL_LES_SMAGORINSKY 1
#define ZL_LES_LEARNED 2
#define ZL_MLP_IN 24
#define ZL_MLP_HIDDEN 64
#define ZL_MLP_TRAINABLE 5825 /* w1 .. b3 */

typedef struct zl_mlp {
    float w1[ZL_MLP_HIDDEN * ZL_MLP_IN];     /* w1[j * 24 + f] */
    float b1[ZL_MLP_HIDDEN];
    float w2[ZL_MLP_HIDDEN * ZL_MLP_HIDDEN]; /* w2[j * 64 + i] */
    float b2[ZL_MLP_HIDDEN];
    float w3[ZL_MLP_HIDDEN];
    float b3;
    float in_mean[ZL_MLP_IN];                /* input normalisation x_hat = (x - mean) * inv_std */
    float in_inv_std[ZL_MLP_IN];
} zl_mlp;

/* Network used by levels with les == ZL_LES_LEARNED (copied; NULL returns to Smagorinsky). */
int zl_set_closure(zl_ctx* ctx, const zl_mlp* net);

/* Run the network on every `every`-th step of a level only (default 1: every step); the steps in
   between relax with each node's c from the last evaluation.  Amortises the network's cost. */
int zl_set_closure_interval(zl_ctx* ctx, int every);

/* The 24 closure features of every node of a full-box level (device array, box order, n * 24). */
int zl_closure_features(zl_ctx* ctx, int level, float* x_device);

/* Box filter of a full-box level over factor^3 blocks of nodes: per block (box order of the
   blocks) 29 FP32 values: rho, u (3), <u_a u_b> (xx yy zz xy xz yz), <f - feq> (19). */
int zl_filter_level(zl_ctx* ctx, int level, int factor, float* out_device);

/* Training pairs on the filtered (coarse) periodic grid of nc[0] x nc[1] x nc[2] blocks:
   target y = c / 0.01 of the least-squares Smagorinsky constant of the exact subgrid stress over
   each 3^3 neighbourhood (clipped to [0, 8]); features of a coarse node holding
   feq(<rho>, <u>) + r <f - feq>, r = factor * tau_eff / tau_fine, tau_eff = tau_coarse + 3 c |S|.
   x_device: n * 24, y_device: n; scratch_device: n * 3 floats. */
int zl_closure_pairs(const int32_t nc[3], const float* filtered_device, double tau_fine, double tau_coarse,
                     int factor, float* x_device, float* y_device, float* scratch_device, void* stream);

/* Network outputs y for n feature rows (device arrays; tensor-core forward of the closure). */
int zl_mlp_forward(const zl_mlp* net, const float* x_device, int64_t n, float* y_device, void* stream);

/* Trainer: FP32 master weights and Adam moments on the device; each step runs the fused
   forward + backward tensor-core kernel over n samples (mean-square error on y) and one Adam
   update (beta1 0.9, beta2 0.999, eps 1e-8). */
typedef struct zl_trainer zl_trainer;
int zl_trainer_create(const zl_mlp* init, int device, zl_trainer** out);
int zl_trainer_set_stream(zl_trainer* tr, void* stream); /* cudaStream_t to issue on (NULL: own stream) */
int zl_trainer_step(zl_trainer* tr, const float* x_device, const float* y_device, int64_t n, float lr);
int zl_trainer_loss(zl_trainer* tr, double* loss);       /* mean-square error of the last step */
int zl_trainer_gradients(zl_trainer* tr, zl_mlp* grad); /* gradients of the last step (w1 .. b3) */
int zl_trainer_weights(zl_trainer* tr, zl_mlp* out);
void zl_trainer_destroy(zl_trainer* tr);

#ifdef __cplusplus
}
#endif
#endif /* ZLLBM_B200_H_ */
