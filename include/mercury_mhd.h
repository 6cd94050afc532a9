/* C ABI of the B200 multi-fluid Hall-MHD step (libmercury_mhd.so).
 *
 * The library replaces the body of the reference's explicit step,
 * MercurySolver::StepOnce() (Z4_Mercury/src/MercurySolver_Driver.cpp:21-61),
 * and its derived-field refresh UpdateDerivedFields_()
 * (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:309-321).  The reference has
 * no plugin or FFI layer; its seam is the C++ class interfaces the step uses:
 *   Field::field(fid, ib) / FieldBlock::operator()(i,j,k,m)
 *       (include/3_field/Field.h:45-52, include/3_field/FieldBlock.h:38-49)
 *       -> mhd_upload_field / mhd_download_field, same index space and layout;
 *   MercuryBoundary::Sync(group) (Z4_Mercury/include/1_Boundary.h:32) and
 *   Halo::sync_group / sync_owner_alias_group (include/4_halo/Halo.h:28-37)
 *       -> mhd_sync_tables (flattened halo and owner copies per group);
 *   ReduceEdgeAliasCandidatesToOwners_ (Z4_Mercury/src/physics/MercurySolver_Current.cpp:3-57)
 *       -> mhd_alias_classes;
 *   calc_physical_constant (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:3-48)
 *       -> mhd_constants.
 *
 * Conventions: plain C types only; every call returns an int status
 * (MHD_OK = 0) and never exits or throws — the reference's exit(-1) on dt
 * underflow (Z4_Mercury/src/physics/MercurySolver_Timestep.cpp:129-140) becomes
 * MHD_ERR_DT, its KSP failure throw becomes MHD_ERR_SOLVE.  A context owns one
 * CUDA stream; calls on one context are synchronous with respect to the host
 * unless stated, and a context is not shared between host threads.
 */
#ifndef MERCURY_MHD_H
#define MERCURY_MHD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum mhd_status {
  MHD_OK = 0,
  MHD_ERR_ARG = 1,      /* invalid argument */
  MHD_ERR_CUDA = 2,     /* CUDA runtime error (see mhd_last_error) */
  MHD_ERR_OOM = 3,      /* device allocation failed */
  MHD_ERR_DT = 4,       /* dt non-finite or below 1e-7 (reference aborts) */
  MHD_ERR_NONFINITE = 5,/* a NaN/Inf in an owned cell's state: the solve is retired
                           at its next step, the batch's other solves go on */
  MHD_ERR_SOLVE = 6,    /* implicit solve did not converge */
  MHD_ERR_STATE = 7,    /* call out of order (e.g. step before prepare) */
  MHD_ERR_TIMEOUT = 8   /* a tile's staged copies did not complete within the fluid
                           kernel's bounded wait (TMA-staged variant): the solve stops */
};

/* Field identifiers: the reference's catalog names
 * (Z4_Mercury/include/0_MercuryFieldCatalog.h:70-202 and the geometry fields of
 * src/7_metric/Metric.cpp:14-73).  ncomp / location in mhd_field_info(). */
enum mhd_field {
  /* state */
  MHD_U_H = 0, MHD_U_NA, MHD_B_XI, MHD_B_ETA, MHD_B_ZETA,
  /* derived (refreshed by the step) */
  MHD_PV_H, MHD_PV_NA, MHD_U_PLUS, MHD_B_CELL, MHD_BIND_CELL, MHD_J_CELL,
  MHD_J_XI, MHD_J_ETA, MHD_J_ZETA,
  /* work (readable for diagnostics) */
  MHD_E_XI, MHD_E_ETA, MHD_E_ZETA, MHD_EHALL_XI, MHD_EHALL_ETA, MHD_EHALL_ZETA,
  MHD_EFACE_XI, MHD_EFACE_ETA, MHD_EFACE_ZETA, MHD_EHC, MHD_HALL_BETA,
  MHD_UCON,                                   /* contravariant U_plus components along xi, eta, zeta */
  MHD_DIVB,                                   /* div B per cell (mhd_div_b) */
  MHD_FNORM_XI, MHD_FNORM_ETA, MHD_FNORM_ZETA, /* unit normal (3) and |JD| of the faces, set by mhd_prepare */
  MHD_PE_NODE,                                /* electron pressure at the nodes: 8-cell mean of p_H + p_Na (ambipolar) */
  MHD_AMBI_COEF,                              /* 9 cell-averaged JD / Jac coefficients of grad p_e, set by mhd_prepare */
  MHD_DPE,                                    /* grad p_e term of the ion momentum sources per cell (ambipolar) */
  MHD_UCON_COEF,                              /* cell-averaged JD (3 x 3) and 1 / (|Jac| + 1e-30) of UCON, set by mhd_prepare */
  MHD_HALL_IH_XI, MHD_HALL_IH_ETA, MHD_HALL_IH_ZETA, /* Hall diffusion length / area ratios (2 per edge), set by mhd_prepare */
  MHD_FLUX_METRIC,                            /* JD of the xi, eta, zeta faces (3 x 3) and 1 / Jac in the step's real type, set by mhd_prepare */
  /* static geometry and sources (uploaded once) */
  MHD_JAC, MHD_JDXI, MHD_JDET, MHD_JDZE, MHD_AREA_XI, MHD_AREA_ETA, MHD_AREA_ZETA,
  MHD_DL_XI, MHD_DL_ETA, MHD_DL_ZETA, MHD_DR_XI, MHD_DR_ETA, MHD_DR_ZETA,
  MHD_HODGE_FACE_XI, MHD_HODGE_FACE_ETA, MHD_HODGE_FACE_ZETA,      /* beta = |l*|/|S| */
  MHD_HODGE_EDGE_XI, MHD_HODGE_EDGE_ETA, MHD_HODGE_EDGE_ZETA,      /* alpha = |e|/|S*| */
  MHD_BCELL_W, MHD_JCELL_W, MHD_BADD_XI, MHD_BADD_ETA, MHD_BADD_ZETA, MHD_PHOTO,
  MHD_CELL_X, MHD_CELL_Y, MHD_CELL_Z,                              /* cell centres */
  MHD_TAPER_XI, MHD_TAPER_ETA, MHD_TAPER_ZETA,                     /* Hall radial taper per edge */
  MHD_TAPER_CELL,                                                  /* Hall radial taper at cell centres (singular edges) */
  MHD_LOCAL_ETA_XI, MHD_LOCAL_ETA_ETA, MHD_LOCAL_ETA_ZETA,         /* local artificial resistivity per edge */
  MHD_ETA_RES_XI, MHD_ETA_RES_ETA, MHD_ETA_RES_ZETA,               /* implicit resistivity per owned edge */
  /* work of the implicit resistive solve (3 components: xi, eta, zeta edges;
   * BSTAR: xi, eta, zeta faces) */
  MHD_RES_W, MHD_RES_X, MHD_RES_R, MHD_RES_P, MHD_RES_Q, MHD_RES_BSTAR,
  MHD_NUM_FIELDS
};

enum mhd_location { MHD_CELL = 0, MHD_FACE_XI, MHD_FACE_ETA, MHD_FACE_ZETA, MHD_EDGE_XI, MHD_EDGE_ETA, MHD_EDGE_ZETA,
                    MHD_NODE };

/* Sync groups: MercuryBoundary::Sync names (Z4_Mercury/src/boundary/Boundary_Build.cpp:564-703).
 * MHD_SYNC_ERES and MHD_SYNC_DB are the implicit resistive substep's Sync("Eres")
 * and Sync("dB") (Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:321,440): the
 * engine keeps E_res in the E edge arrays and dB in the B face arrays, so their
 * tables address those fields; they differ from MHD_SYNC_EEDGE and MHD_SYNC_BFACE
 * only in the physical handlers (Farfield: copy, Coupled-Solid: nothing).  dJ
 * (in the J edge arrays) shares MHD_SYNC_JEDGE's handlers and tables.  Only
 * solves with the implicit resistive substep read them.  MHD_SYNC_BADD is
 * Sync("Badd") of the background field (Z4_Mercury/src/MercurySolver.cpp:141),
 * run once after the background is set (mhd_setup_geometry_bg); periodic
 * blocks and lattices have no copies in it. */
enum mhd_group { MHD_SYNC_UCELL = 0, MHD_SYNC_BFACE, MHD_SYNC_EHALL, MHD_SYNC_EEDGE, MHD_SYNC_B_CELL,
                 MHD_SYNC_JEDGE, MHD_SYNC_J_CELL, MHD_SYNC_ERES, MHD_SYNC_DB, MHD_SYNC_BADD, MHD_NUM_GROUPS };

/* Indices into mhd_constants.bc (BuildMercuryBackgroundState,
 * Z4_Mercury/include/0_BackgroundState.h:18-85, and the wall floors of
 * BC_Solid_Surface_) */
enum mhd_bc_const {
  MHD_BC_QINF = 0,        /* 5: upstream H+ conserved state */
  MHD_BC_QINFS = 5,       /* 5: upstream Na+ conserved state */
  MHD_BC_BIMF = 10,       /* 3: IMF */
  MHD_BC_ZERO = 13,       /* 0.0 */
  MHD_BC_NA_RHO_FLOOR = 14, /* 1e-12 */
  MHD_BC_NA_E_FLOOR = 15, /* 1e-12 / (gamma - 1) */
  MHD_BC_UINF = 16,       /* 3: upstream velocity */
  MHD_NUM_BC = 19
};

/* Physical constants as calc_physical_constant derives them (Tools.cpp:3-48). */
typedef struct mhd_constants {
  double gamma, M_H, M_Na, M_ref, T_ref, L_ref, U_ref, B_ref, n_ref, rho_ref, m_Na, k_Boltz, q_e, mu0;
  double state_coeff_H, state_coeff_Na, CFL, hall_coef, momentum_induce_coeff, momentum_hall_coeff;
  double inver_MA2, ne_hall_floor;
  /* artificial resistivity (AddArtificialResistivityToEdgeEMF_,
   * Z4_Mercury/src/physics/MercurySolver_MagExplicit_Resis.cpp:6-64):
   * E += eta_art(|J|/|dr|) J with eta_art rising smoothly from 0 at
   * arti_J_start to arti_eta_max at arti_J_on; off when arti_eta_max <= 0 */
  double arti_eta_max, arti_J_start, arti_J_on;
  int32_t ambipolar;  /* is_Ambipolar_Efield */
  int32_t local_arti; /* E += MHD_LOCAL_ETA * J (AddLocalArtificialResistivityToEdgeEMF_, same file :66-185) */
  /* implicit resistive substep (SolveImplicitResistiveDiffusion_,
   * Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:475-555): after the
   * explicit update, solve (I + dt eta alpha C^T beta C) E = eta J(B*) on the
   * owned edges with eta > 0 (eta: MHD_ETA_RES_*), then B = B* - dt curl E.
   * Solved to ||A E - b|| <= res_rtol ||b||, else MHD_ERR_SOLVE.  FP64
   * solves: preconditioned CG (at most res_max_it iterations, capped at
   * 100000; res_rtol 0 = 1e-13), its iteration loop run on the device as a
   * CUDA graph with a conditional loop node.  Mixed-precision solves
   * (res_rtol 0 = 1e-10) on the solve's FP64 companion fields: while the
   * previous substep took at most res_direct_iters iterations, FP64 CG there;
   * after a longer one, iterative refinement with the residual A E - b and
   * its norms in FP64 and each correction solved by FP32 CG (on the solve's
   * own FP32 edge fields) to 1e-4 of its right-hand side (at most res_max_it
   * iterations each, at most 30 refinements). */
  double res_rtol;
  int32_t resistive;  /* is_Mercury_resistance */
  int32_t res_max_it;
  /* values of the physical boundary operations (mhd_bc_const) */
  double bc[MHD_NUM_BC];
  int32_t res_direct_iters; /* 0 = 20; negative: always iterative refinement */
  int32_t pad_;
} mhd_constants;

/* One DOF reference in the FieldBlock index space. */
typedef struct mhd_dof {
  int32_t field, block, i, j, k, comp;
} mhd_dof;

/* One flattened copy dst <- sign * src.  A group's halo copies are applied
 * first (all reading pre-sync values), then its owner copies, exactly the
 * stage order of MercuryBoundary::Sync_ (Z4_Mercury/src/boundary/Boundary_Sync_.cpp:4-110). */
typedef struct mhd_copy {
  mhd_dof dst, src;
  double sign;
} mhd_copy;

/* Physical boundary operations of a sync group (BoundaryCore::ApplyPhysical
 * with the handlers MercuryBoundary::InstallHandlers registers,
 * Z4_Mercury/src/boundary/Boundary_Build.cpp:5-300), run before the group's
 * copies.  The copies of a boundary handler (ghost <- boundary layer) are
 * ordinary entries of the group's halo table; these are the operations that
 * compute a value:
 *   MHD_PHYS_SET   dst <- mhd_constants.bc[arg] (farfield states, IMF, floors, zero)
 *   MHD_PHYS_WALL  the solid-wall state of BC_Solid_Surface_
 *                  (Z4_Mercury/src/boundary/Boundary_Condition_Fluid.cpp:37-259) on the
 *                  five components of cell dst from cell src (one cell deeper
 *                  in the fluid), then on the nghost ghost cells outward of
 *                  dst along direction arg (+-1, +-2, +-3), clamped to the
 *                  allocated range
 *   MHD_PHYS_EFAR  edge dst <- E_inf . dr(dst), E_inf = -u_inf x B_imf
 *                  (BC_Farfield_Eedge_set_zerocurl,
 *                  Z4_Mercury/src/boundary/Boundary_Condition.cpp:573-624) */
enum mhd_phys_kind { MHD_PHYS_SET = 0, MHD_PHYS_WALL = 1, MHD_PHYS_EFAR = 2 };
typedef struct mhd_phys_op {
  int32_t kind, arg;
  mhd_dof dst, src;
} mhd_phys_op;

/* A pseudo field of mhd_dof: slot `i` of the solve's staging area.  A sync
 * copy whose source the same copy phase overwrites (the reference's halo
 * exchange packs every source before it writes, src/4_halo/component_copy/
 * HaloExchangeInner.cpp:93-160) goes through a staging slot. */
#define MHD_STAGING 1000

typedef struct mhd_sync_group {
  int32_t n_halo, n_owner;
  const mhd_copy *halo;
  const mhd_copy *owner;
  int32_t n_phys, n_stash;
  const mhd_phys_op *phys;   /* physical boundary operations, run first */
  const mhd_copy *stash;     /* 2 n_stash entries: n_stash copies staging <- source (after the
                                physical operations), then n_stash copies destination <- staging
                                (after the halo copies) */
} mhd_sync_group;

/* Edge alias classes (global_id order): class c has members
 * member[offset[c] .. offset[c+1]) with orientation signs, written to
 * owner[c] as owner_sign * (sum_m sign_m * value_m) / count. */
typedef struct mhd_alias_classes {
  int32_t n_classes;
  const int32_t *offset;      /* n_classes + 1 */
  const mhd_dof *member;      /* offset[n_classes] (field = location axis 0/1/2) */
  const double *member_sign;
  const mhd_dof *owner;       /* n_classes */
  const double *owner_sign;
} mhd_alias_classes;

/* Singular (valence-3) physical edges of a multi-block grid
 * (SingularEdgeRegistry, src/7_metric/SingularEdgeRegistry.cpp:78-332): the
 * owner edge of each, its aliases (for the mean length and the canonical
 * edge vector), the incident cells (EMF and Hall EMF: weighted by |Jac|) and
 * the incident owner faces (the current).  Weights, the canonical vector and
 * the inverse Hodge star are computed on the device from the uploaded
 * geometry when the solve is prepared. */
typedef struct mhd_singular_alias {
  mhd_dof edge;       /* field = edge axis 0/1/2 */
  int32_t orient, pad_;
} mhd_singular_alias;
typedef struct mhd_singular_cell {
  mhd_dof cell;
  int32_t axis, orient; /* axis and orientation of the alias the cell was reached from */
} mhd_singular_cell;
typedef struct mhd_singular_face {
  mhd_dof face;         /* field = face axis 0/1/2 */
  int32_t sign, pad_;   /* incidence sign x alias orientation (0: no contribution) */
} mhd_singular_face;
typedef struct mhd_singular_edges {
  int32_t n_edges;
  const mhd_dof *owner;             /* field = edge axis 0/1/2 */
  const double *owner_sign;
  const int32_t *alias_offset;      /* n_edges + 1 */
  const mhd_singular_alias *aliases;
  const int32_t *cell_offset;       /* n_edges + 1 */
  const mhd_singular_cell *cells;
  const int32_t *face_offset;       /* n_edges + 1 */
  const mhd_singular_face *faces;
} mhd_singular_edges;

typedef struct mhd_desc {
  int32_t n_blocks;
  const int32_t *cells;   /* n_blocks * 3: cells per axis (mx, my, mz) */
  int32_t nghost;         /* runtime ghost width ngg (4 in production) */
  int32_t precision;      /* 0 = FP64 (parity path); 1 = mixed (FP32 state/flux, FP64 metric Jac/JD) */
  mhd_constants constants;
  mhd_sync_group groups[MHD_NUM_GROUPS];
  mhd_alias_classes edge_aliases;
  /* multi-block grids with physical boundaries (zero / NULL otherwise) */
  int32_t n_staging;               /* staging slots the groups' stash copies use */
  int32_t n_wall;
  const mhd_phys_op *wall;         /* the step's wall EMF: E_t = 0 on solid-wall edges
                                      (ApplyStationaryWallNonResistiveEMF_,
                                      Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:5-88) */
  mhd_singular_edges singular;
} mhd_desc;

typedef struct mhd_ctx mhd_ctx;
typedef struct mhd_batch mhd_batch; /* many solves on one GPU: see "batched solves" below */

/* Replaces the MercurySolver constructor's device-side duties: allocates the
 * device field arena (SoA, one array per component), uploads the sync and
 * alias tables.  Fields are uploaded separately. */
int mhd_ctx_create(const mhd_desc *desc, mhd_ctx **out);
int mhd_ctx_destroy(mhd_ctx *ctx);

/* Field::field(fid, ib) data exchange.  `data` is the FieldBlock storage of
 * that field: AoS, offset ((i-lo0)*e1 + (j-lo1))*e2*ncomp + (k-lo2)*ncomp + m
 * (include/3_field/FieldArray.h:126-128), for the logical range [lo, hi). */
int mhd_upload_field(mhd_ctx *ctx, int field, int block, const double *data, const int32_t lo[3],
                     const int32_t hi[3], int ncomp);
int mhd_download_field(mhd_ctx *ctx, int field, int block, double *data, const int32_t lo[3],
                       const int32_t hi[3], int ncomp);
/* Sets every position of [lo, hi) to values[m] per component m (ncomp <= 36)
 * on the device: a uniform state without its host array (Common_Initial,
 * Z4_Mercury/include/2_Initial.h:134-215, sets U and B that way). */
int mhd_fill_field(mhd_ctx *ctx, int field, int block, const double *values, const int32_t lo[3],
                   const int32_t hi[3], int ncomp);
/* mhd_batch_set_constants of the context's solve. */
int mhd_set_constants(mhd_ctx *ctx, const mhd_constants *constants);

/* The preamble of MercurySolver::Advance (Z4_Mercury/src/MercurySolver_Driver.cpp:6-13):
 * UpdateDerivedFields_ on the uploaded state.  Sets time/step. */
int mhd_prepare(mhd_ctx *ctx, double time, int64_t step);

/* nsteps calls of StepOnce.  dt_out (optional) receives the last dt.  The
 * steps are captured once into a CUDA graph and replayed. */
int mhd_step(mhd_ctx *ctx, int nsteps, double *dt_out);

/* Same as mhd_step but returns without waiting for the GPU (status is
 * checked on the next synchronous call). */
int mhd_step_async(mhd_ctx *ctx, int nsteps);
int mhd_synchronize(mhd_ctx *ctx);

/* Profiling form of mhd_step (no graph): runs nsteps steps eagerly with a
 * CUDA event after every kernel and returns, per kernel launch of one step
 * (in launch order), its mean duration in ms and its name.  The reference
 * has no counterpart (its only timer is RuntimeMonitor's CPU time per step,
 * src/6_io/RuntimeMonitor.cpp:33-56). */
int mhd_step_profiled(mhd_ctx *ctx, int nsteps, int max_kernels, float *kernel_ms, const char **kernel_names,
                      int *n_kernels);

/* MercuryBoundary::Sync(group) on device data. */
int mhd_sync(mhd_ctx *ctx, int group);

typedef struct mhd_info {
  double time, dt;
  int64_t step;
  int32_t status;      /* sticky device status (mhd_status) */
  int32_t pad_;
  int64_t device_bytes;
  int64_t remaining;   /* steps of the current request not yet taken */
  /* last implicit resistive substep of the solve (zeros without one):
   * residual norm / ||b|| at exit (FP64 solves: CG's recursive residual;
   * mixed precision: the refinement's FP64 residual ||A E - b||), CG
   * iterations (over all refinements) and refinements (0 in FP64 solves) */
  double res_relres;
  int32_t res_iters, res_refinements;
} mhd_info;
int mhd_get_info(mhd_ctx *ctx, mhd_info *info);
/* The solve's sticky device status (an mhd_status: MHD_OK, or the first
 * failure a step met, e.g. MHD_ERR_DT where the reference exits,
 * Z4_Mercury/src/physics/MercurySolver_Timestep.cpp:139, or MHD_ERR_SOLVE
 * where it throws, Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:520),
 * after the work queued so far.  Returns MHD_OK when the status was read. */
int mhd_get_status(mhd_ctx *ctx, int32_t *status);

/* calc_divB (Z4_Mercury/src/physics/MercurySolver_MagneticCell.cpp:151-241) on
 * the current state: MHD_DIVB = (sum of the cell's outward face fluxes) / Jac
 * on the owned cells, and *max_abs = max |div B| over them.  (The reference
 * zeroes the first shell next to "Pole" patches; blocks built from
 * mhd_topology_periodic_block have none.) */
int mhd_div_b(mhd_ctx *ctx, double *max_abs);
int mhd_batch_div_b(mhd_batch *batch, int slot, double *max_abs);

/* Static description of a field id: ncomp and mhd_location. */
int mhd_field_info(int field, int32_t *ncomp, int32_t *location);

/* CUDA stream the context runs on (cudaStream_t as void*). */
void *mhd_stream(mhd_ctx *ctx);

/* Number of kernels one mhd_step(ctx, 1) launches (for launch accounting). */
int mhd_kernels_per_step(mhd_ctx *ctx);

/* Raw device pointer of one field component array of a block, with the box
 * layout: element (i,j,k) at base[(i+G)*si + (j+G)*sj + (k+G)].  The
 * elements are double, except in mixed precision (mhd_desc.precision = 1),
 * where every field other than MHD_JAC and MHD_JD* holds float. */
int mhd_device_view(mhd_ctx *ctx, int field, int block, int comp, double **base, int32_t *G, int64_t *si,
                    int64_t *sj, int32_t ext[3]);

/* Seeded uniform draws of the synthetic workloads (host only): std::mt19937_64
 * seeded with `seed`, u = (x >> 11) * 2^-53, out[t] = -a + 2 a u in draw order.
 * No counterpart in the reference solver; it reproduces the seeding the
 * workload definition states, so that host-generated initial states are
 * byte-identical to the ones the CPU oracle generates. */
int mhd_seeded_uniform(uint64_t seed, int64_t count, double a, double *out);

/* Host helpers of the cubed-sphere shell case: the nodes of panel `panel`
 * over [-G, n + 1 + G) per axis (AoS, k fastest).  The owned
 * nodes are the equiangular panel directions (panels 0-3 around the z axis,
 * 4 north, 5 south) at radii r_k = r_out^(k / nr); the reference reads them
 * from grid files, so they have no counterpart there.  The ghost nodes are
 * extrapolated as the reference's grid reader adds them (Block::Add_ghostmesh,
 * src/1_grid/1_MPCNS_Grid.cpp:591-815), so the static fields computed from
 * them match the reference's on every position it fills.  And the Hall radial
 * taper (HallRadialTaper_, Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:6-13)
 * at n points. */
int mhd_shell_nodes(int32_t na, int32_t nr, double r_out, int32_t panel, int32_t G, double *out);
/* All six panels' nodes (panel-major, each as mhd_shell_nodes lays it out)
 * with the ghost nodes the reference's grid preprocessing leaves on this
 * grid (Grid::Grid_Preprocess, include/1_grid/1_MPCNS_Grid.h:151-224:
 * extrapolation, the inner-interface mesh transfer and the corner
 * treatment): the strips beside a panel edge hold the neighbour panel's
 * nodes, the corner columns the nodes those strips received.  G <= na. */
int mhd_shell_grid(int32_t na, int32_t nr, double r_out, int32_t G, double *out);
int mhd_hall_taper(double r_min, double r_max, int64_t n, const double *xyz, double *out);

/* ---- Hall edge EMF without device allocation ----
 * No counterpart in the reference: it exists for callers that may not call
 * cudaMalloc / cudaFree themselves (a host framework that owns all device
 * memory through its own pool, or a request loop that must not allocate per
 * call).  The caller passes device pointers to its inputs and outputs in the
 * box layout of mhd_device_view (element (i,j,k) at p[(i+G)*si + (j+G)*sj +
 * (k+G)], G >= nghost + 1, sj >= n[2] + 1 + 2G, si >= sj (n[1] + 1 + 2G));
 * the only intermediate — alpha (J x B) and |alpha||B| on the cells
 * [-1, n]^3 around the owned edges — lives in a library-owned static device
 * array of MHD_HALL_SCRATCH_MAX_CELLS cells x 4 doubles (32 MiB), held by
 * every GPU that loads the library until the process exits.  Blocks with
 * (n[0] + 2)(n[1] + 2)(n[2] + 2) above that, and strides smaller than the
 * box, return MHD_ERR_ARG with a message (mhd_last_error).  The first call on a
 * device looks up the array's device address (once per device, with that
 * device current); make that first call before any stream capture.  All calls
 * share the one array and nothing in it needs to start at zero (every cell is
 * written before it is read), but calls that overlap on the GPU race on it:
 * serialise them (one stream, or one device at a time).  Writes the Hall EMF
 * on the owned edges of all three families; launches asynchronously on
 * `stream` (cudaStream_t as void*; NULL = default stream). */
#define MHD_HALL_SCRATCH_MAX_CELLS (1 << 20)
typedef struct mhd_hall_block {
  int32_t n[3];        /* cells per axis */
  int32_t nghost;      /* runtime ghost width (4) */
  int32_t G;           /* box ghost width of the pointers (>= nghost + 1) */
  int32_t pad_;
  int64_t si, sj;      /* box strides (k contiguous) */
  const double *rho_H, *rho_Na;                  /* U_H and U_Na component 0 (cells) */
  const double *J_cell[3], *B_cell[3];           /* cells */
  const double *B_face[3];                       /* induced face fluxes xi, eta, zeta */
  const double *area[3];                         /* |S| of xi, eta, zeta faces */
  const double *dl[3];                           /* |e| of xi, eta, zeta edges */
  const double *dr_xi[3], *dr_eta[3], *dr_zeta[3];/* edge vectors, x/y/z components */
  const double *taper[3];                        /* Hall radial taper per edge */
  double hall_coef, M_H, M_Na, M_ref, ne_hall_floor;
} mhd_hall_block;
int mhd_hall_emf_static_scratch(const mhd_hall_block *in, double *out_xi, double *out_eta, double *out_zeta,
                                void *stream);

/* ---- batched solves (ensembles and request serving) ----
 * No counterpart in the reference, which runs one solve per MPI job.  A batch
 * holds up to `capacity` independent solves (slots) on one GPU and advances
 * all of them with one CUDA graph per step: every kernel of the step is a
 * persistent loop over the tiles of all active slots, so one launch covers
 * every member and the graph stays valid while slots join and leave.  A slot
 * is active while it has steps left in its request; slots with different
 * block shapes, sync tables and constants share a batch.  mhd_ctx is a batch
 * of capacity 1.  Calls on one batch are serialised by the caller. */
/* precision: 0 = FP64 (every field double); 1 = mixed (state, work and
 * static fields float, fluxes / EMFs / updates computed in float; the metric
 * MHD_JAC and MHD_JD* stays double).  Every solve of a batch has the batch's
 * precision (mhd_desc.precision).  Uploads and downloads always exchange
 * doubles; mhd_batch_device_view returns a float array for float fields. */
int mhd_batch_create(int capacity, int precision, mhd_batch **out);
int mhd_batch_destroy(mhd_batch *batch);
/* Grows the batch's device memory pool by `bytes` ahead of the solves that
 * will use it (the pool keeps memory that solves free, and memory reserved
 * here, until mhd_batch_destroy): solves added later take their arenas and
 * tables from it without mapping new memory.  No reference counterpart (its
 * solver allocates at setup).  Synchronous. */
int mhd_batch_reserve(mhd_batch *batch, int64_t bytes);
/* Device bytes a solve of this descriptor occupies (arena and tables, and
 * for a mixed-precision solve with the implicit resistive substep its FP64
 * companion, which holds the refinement's residual); -1 on a bad descriptor.
 * Lets a server admit requests against free HBM. */
int64_t mhd_desc_device_bytes(const mhd_desc *desc);
/* Adds a solve (allocates its arena, uploads its tables) into a free slot;
 * stream-ordered with the batch's other work. */
int mhd_batch_add(mhd_batch *batch, const mhd_desc *desc, int *slot);
/* Adds a one-block solve periodic in every direction (cells, nghost and the
 * constants as in mhd_desc; the batch's precision) with its sync tables and
 * edge alias classes compiled directly from the periodic connectivity, the
 * same copies mhd_topology_periodic_block lists (no explicit copy lists:
 * the fast way to admit such a solve).  No reference counterpart (its
 * topology builder, src/2_topology/TopologyBuilder.cpp:436, makes the lists). */
int mhd_batch_add_periodic(mhd_batch *batch, const int32_t cells[3], int32_t nghost, const mhd_constants *constants,
                           int *slot);
/* Adds a solve with the blocks and topology of the solve in src_slot, sharing
 * its device sync and alias tables (no descriptor processing): the way a
 * server admits a request whose grid it already holds.  constants: the new
 * solve's constants (NULL = the template's).  copy_static = 1 copies the
 * template's fields (static geometry, sources, and its current state) on
 * the device; 0 zeroes them.  The caller then uploads what differs (normally
 * the state) and calls mhd_batch_sync / mhd_batch_prepare as after
 * mhd_batch_add. */
int mhd_batch_add_like(mhd_batch *batch, int src_slot, const mhd_constants *constants, int copy_static, int *slot);
/* Frees a slot; the solve's memory is released in stream order. */
int mhd_batch_remove(mhd_batch *batch, int slot);
int mhd_batch_upload_field(mhd_batch *batch, int slot, int field, int block, const double *data,
                           const int32_t lo[3], const int32_t hi[3], int ncomp);
int mhd_batch_download_field(mhd_batch *batch, int slot, int field, int block, double *data,
                             const int32_t lo[3], const int32_t hi[3], int ncomp);
int mhd_batch_fill_field(mhd_batch *batch, int slot, int field, int block, const double *values,
                         const int32_t lo[3], const int32_t hi[3], int ncomp);
/* Replaces a solve's constants (a new upstream state on the same grid: the
 * parameter lists calc_physical_constant and BuildMercuryBackgroundState read,
 * Z4_Mercury/src/physics/MercurySolver_Tools.cpp:3-48); the implicit substep's
 * presence must not change.  mhd_batch_prepare must follow. */
int mhd_batch_set_constants(mhd_batch *batch, int slot, const mhd_constants *constants);
int mhd_batch_sync(mhd_batch *batch, int slot, int group);
int mhd_batch_prepare(mhd_batch *batch, int slot, double time, int64_t step);
/* The fluid kernel's tile variants (Scheme_U_ + sources + update, the
 * step's largest pass): variant v tiles the owned cells in CTAs of 256
 * threads, shape[0] x shape[1] x shape[2] cells along k, j, i, compiled for
 * shape[3] resident CTAs per SM (its register cap).  A batch runs one
 * (default 0); mhd_batch_time_fluid_tiles times each on the batch's active
 * solves (the fluid pass alone, `reps` launches after one untimed, writing
 * only the next-step state buffer, which the next step rewrites: the solves'
 * results do not change), mhd_batch_fluid_tile sets one (the step graphs are
 * captured anew).  The choice does not change results: every variant
 * computes each face flux and cell update with the same operations.
 * Variant 6 (16 x 4 x 4) stages each tile's cells with TMA tensor copies,
 * the next tile's while the current one is computed. */
#define MHD_NUM_FLUID_TILES 7
int mhd_fluid_tile_shape(int variant, int32_t shape[4]);
int mhd_batch_fluid_tile(mhd_batch *batch, int variant);
int mhd_batch_time_fluid_tiles(mhd_batch *batch, int reps, float ms[MHD_NUM_FLUID_TILES]);
int mhd_fluid_tile(mhd_ctx *ctx, int variant);  /* mhd_batch_fluid_tile of a context */
/* Sets the slot's request to nsteps more steps (0 parks it). */
int mhd_batch_request(mhd_batch *batch, int slot, int64_t nsteps);
/* Enqueues nsteps graph launches of the batched step (asynchronous).  Each
 * launch advances every slot that still has steps requested by one step. */
int mhd_batch_run(mhd_batch *batch, int nsteps);
/* Mean device time per step of the implicit resistive substep (every
 * resistive solve at once: prologue, CG loop, epilogue) over the steps run
 * since the previous call, in ms (0 when none ran); waits for the batch's
 * stream and restarts the count. */
int mhd_batch_substep_ms(mhd_batch *batch, double *ms_per_step);
/* on != 0: the substep's CG iterations are launched one by one from the host
 * (the same kernels and results, a host round trip per iteration) instead of
 * the device loop, for profilers that do not follow conditional graph nodes.
 * Off by default. */
int mhd_batch_cg_host_loop(mhd_batch *batch, int on);
/* Synchronises and fills infos[0 .. capacity) (empty slots read zero). */
int mhd_batch_poll(mhd_batch *batch, mhd_info *infos);
/* Asynchronous form: mhd_batch_poll_async enqueues a snapshot of every slot's
 * state after the work queued so far and returns a ticket (two snapshots can
 * be outstanding); mhd_batch_poll_wait waits for that snapshot only, so the
 * host can act on step k while step k + 1 runs.  Uploads from pageable host
 * memory, mhd_batch_add_like, mhd_batch_sync, mhd_batch_prepare,
 * mhd_batch_request and mhd_batch_remove are asynchronous too (stream-ordered
 * with the steps). */
int mhd_batch_poll_async(mhd_batch *batch, int *ticket);
int mhd_batch_poll_wait(mhd_batch *batch, int ticket, mhd_info *infos);
void *mhd_batch_stream(mhd_batch *batch);
int mhd_batch_kernels_per_step(mhd_batch *batch);
int mhd_batch_step_profiled(mhd_batch *batch, int nsteps, int max_kernels, float *kernel_ms,
                            const char **kernel_names, int *n_kernels);
int mhd_batch_device_view(mhd_batch *batch, int slot, int field, int block, int comp, double **base, int32_t *G,
                          int64_t *si, int64_t *sj, int32_t ext[3]);

/* Text of the last error on this thread. */
const char *mhd_last_error(void);

/* ---- host-side topology builders (C++ in the library, no device work) ----
 * Flattened sync tables and edge alias classes for ONE block of n^3 cells,
 * periodic in every direction (the reference's periodic inner patches with
 * negative block ids, src/1_grid/1_MPCNS_Grid.cpp:455-464).  The tables are
 * owned by the returned handle. */
typedef struct mhd_topology mhd_topology;
int mhd_topology_periodic_block(const int32_t cells[3], int32_t nghost, mhd_topology **out);
/* A box periodic in every direction cut into blocks[0] x blocks[1] x
 * blocks[2] aligned blocks of cells[3] cells each, joined face to face
 * (block id (p * blocks[1] + q) * blocks[2] + r for lattice position
 * (p, q, r)): the sync tables and edge alias classes the reference builds
 * for such inner patches (Grid::Read_Inner_Boundary,
 * src/1_grid/1_MPCNS_Grid.cpp:400-517; TopologyBuilder.cpp:436;
 * HaloBuild.cpp:382-540).  A block needs at least nghost cells along every
 * axis.  The descriptor it fills has blocks[0] * blocks[1] * blocks[2]
 * blocks. */
int mhd_topology_periodic_lattice(const int32_t cells[3], const int32_t blocks[3], int32_t nghost,
                                  mhd_topology **out);
/* A general multi-block grid: blocks of cells[3 b .. 3 b + 2] cells, their
 * inner face patches in the reference's topology order
 * (Topology::inner_patches, TOPO::build_topology,
 * src/2_topology/TopologyBuilder.cpp:436; node boxes half-open, the node
 * index map this -> nb: nb[perm[a]] = sign[a] * this[a] + offset[a],
 * src/2_topology/TopologyOps.cpp:77-230) and physical patches
 * (Farfield or the solid wall, Coupled-Solid).  The builder derives the edge
 * and vertex patches as the reference does
 * (src/2_topology/TopologyEdge.cpp:45-345), replays every sync group of
 * MercuryBoundary::Sync (physical handlers, the three halo stages with the
 * reference's exchange rules, owner-to-alias copies;
 * Z4_Mercury/src/boundary/Boundary_Sync_.cpp:4-110) on symbolic DOF values and
 * flattens the result into the descriptor's tables; it also builds the face
 * and edge equivalence classes (owner = smallest (block, i, j, k), canonical
 * orientation from the smallest node representatives,
 * src/2_topology/TopologyQuery.cpp:104-190), the edge alias classes, the
 * singular-edge lists and the wall-EMF edges.  resistive selects the
 * handler set of is_Mercury_resistance. */
typedef struct mhd_patch {
  int32_t this_block, nb_block, direction, nb_direction;
  int32_t this_lo[3], this_hi[3], nb_lo[3], nb_hi[3];
  int32_t perm[3], sign[3], offset[3];
  int32_t dir3;   /* edge and vertex patches: direction, dir2, dir3 are their face directions */
} mhd_patch;
enum mhd_bc_kind { MHD_BC_FARFIELD = 0, MHD_BC_SOLID = 1 };
typedef struct mhd_physical_patch {
  int32_t block, direction, bc, pad_;
  int32_t lo[3], hi[3];
} mhd_physical_patch;
int mhd_topology_multiblock(int32_t n_blocks, const int32_t *cells, int32_t nghost, int32_t n_faces,
                            const mhd_patch *faces, int32_t n_physical, const mhd_physical_patch *physical,
                            int32_t resistive, mhd_topology **out);
/* The 6-panel gnomonic cubed-sphere shell of na x na x nr cells per panel
 * (panel axes: i, j angular, k radial; the panel numbering and patch order
 * of the oracle's shell case): inner sphere k = 0 a solid wall, outer sphere
 * k = nr Farfield, eight valence-3 radial lines. */
int mhd_topology_cubed_sphere(int32_t na, int32_t nr, int32_t nghost, int32_t resistive, mhd_topology **out);
/* The patches a multi-block builder used: which = 0 inner face patches,
 * 1 inner edge patches, 2 inner vertex patches (direction/nb_direction/dir3
 * hold the edge's or vertex's face directions); and the physical patches. */
int mhd_topology_patches(const mhd_topology *topo, int32_t which, const mhd_patch **patches, int32_t *n);
int mhd_topology_physical(const mhd_topology *topo, const mhd_physical_patch **patches, int32_t *n);
int mhd_topology_fill_desc(const mhd_topology *topo, mhd_desc *desc);
int mhd_topology_destroy(mhd_topology *topo);

/* ---- Per-solve setup on the device ----
 * Computes every static field the step reads for one block from its node
 * coordinates, with the reference's formulas (compute_metric_fields,
 * src/7_metric/Metric.cpp:108-669,1261-1328; SetupCellReconstructionWeights_,
 * Z4_Mercury/src/MercurySolver_ReconstructionSetup.cpp:29-193;
 * Initial_Na_And_PhotoRate_, Z4_Mercury/include/2_Initial.h:227-440): JAC,
 * JD*, AREA_*, DL_*, DR_*, HODGE_FACE_*, HODGE_EDGE_*, BCELL_W, JCELL_W,
 * PHOTO, CELL_X/Y/Z; BADD_* zero (no dipole, no IMF) and TAPER_* 1 on the
 * owned edges (Hall radial taper off).  nodes: x, y, z interleaved, (i, j, k)
 * over [-(nghost + 1), n + nghost + 2) per axis, i slowest (AoS, like
 * mhd_upload_field with 3 components).  L_ref: the length unit of the photo
 * rate.  Replaces uploading those fields; the state is uploaded as before.
 * Asynchronous like mhd_batch_upload_field (it waits only for page-locked
 * nodes); mhd_prepare must follow. */
int mhd_batch_setup_geometry(mhd_batch *batch, int slot, int block, const double *nodes, double L_ref);
int mhd_setup_geometry(mhd_ctx *ctx, int block, const double *nodes, double L_ref);

/* The inputs of a magnetosphere case that the reference derives from its
 * parameter lists, for mhd_setup_geometry_bg:
 *   the background field (DipoleField, Z4_Mercury/include/operators/Dipole.h:26-43,
 *     load_from_param :46-86, Build_Badd_FaceFlux :89-363): the dipoles'
 *     vector potential A along the edges [-1, n + stagger] of the block,
 *     integrated as A(midpoint) . dr, its curl on the faces it reaches, plus
 *     B0 . JD of the IMF on every face of [-g, n + stagger + g);
 *   the Hall radial taper (HallRadialTaperEdge_, HallRadialTaper_,
 *     Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:6-25) at the
 *     owned edges' midpoints and the owned cells' centres (0 elsewhere);
 *   the implicit resistivity per owned edge (ImplicitResistiveEtaAtEdge_,
 *     Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:228-253, with
 *     MercuryResistivityShape_, Z4_Mercury/src/physics/MercurySolver_Tools.cpp:50-69),
 *     written when the solve has the implicit substep.
 * The dipoles, IMF and length / field units are in SI as the reference's
 * lists hold them and are nondimensionalised as load_from_param does. */
#define MHD_MAX_DIPOLES 4
typedef struct mhd_background {
  int32_t n_dipoles, pad_;
  double dipole[MHD_MAX_DIPOLES][7]; /* x0 y0 z0 [m], mx my mz [A m^2], a [m]: the Dipole<n> lists */
  double B_imf[3];                   /* Bx By Bz [T] of the INITIAL list */
  double L_ref, B_ref, mu_mag;       /* REF list and mu_mag of the constant list */
  double hall_r_min, hall_r_max;     /* r_min, r_max of the Hall taper (equal: a step at r_min) */
  double inver_Rem;                  /* eta_max_mercury / (mu_mag U_ref L_ref) (calc_physical_constant) */
  double eta_r_inner, eta_r_outer, eta_width; /* mercury_eta_r_inner, _outer, _width */
} mhd_background;
/* mhd_setup_geometry plus the background, taper and resistivity of `bg` on
 * the block (bg NULL: mhd_setup_geometry).  Once every block of the solve is
 * set, mhd_sync / mhd_batch_sync(MHD_SYNC_BADD) completes the background as
 * the reference's Sync("Badd") does. */
int mhd_batch_setup_geometry_bg(mhd_batch *batch, int slot, int block, const double *nodes, double L_ref,
                                const mhd_background *bg);
int mhd_setup_geometry_bg(mhd_ctx *ctx, int block, const double *nodes, double L_ref, const mhd_background *bg);

/* ---- Restart files ----
 * The reference's checkpoint format, MPCNSRST version 1
 * (IOModule::WriteRestartBinFile / ReadRestartBinFile,
 * src/6_io/IOModule_Bin.cpp:168-420), with the fields its Mercury solver
 * checkpoints: U_H, U_Na, B_xi, B_eta, B_zeta
 * (Z4_Mercury/src/MercurySolver.cpp:33-35).  Files written here resume in the
 * reference and the reference's files resume here. */
#define MHD_RESTART_FIELDS 5 /* U_H, U_Na, B_xi, B_eta, B_zeta, in this order */
typedef struct mhd_restart_image {
  int32_t step;          /* steps taken */
  double time;           /* physical time */
  int32_t n_blocks;
  const int32_t *cells;  /* 3 per block */
  int32_t nghost;
  /* per state field: the blocks' arrays one after another, each over the
   * FieldBlock range [-nghost, n + stagger + nghost) in (i, j, k, comp)
   * order (mhd_restart_values doubles in all) */
  double *data[MHD_RESTART_FIELDS];
  uint32_t loaded;       /* mhd_restart_read: bit f set when the file held field f */
} mhd_restart_image;
/* Doubles of state field `state_field` over all blocks; -1 on bad arguments. */
int64_t mhd_restart_values(const mhd_restart_image *img, int32_t state_field);
/* Host-only file I/O of an image.  The reader checks the header, block count,
 * and for the state fields their location, components, nghost and ranges
 * against img (cells, nghost) as the reference's reader does; fields it does
 * not restore are skipped; fields missing from the file are left as they
 * are (see `loaded`).  No device work. */
int mhd_restart_write(const char *path, const mhd_restart_image *img);
int mhd_restart_read(const char *path, mhd_restart_image *img);
/* Writes a solve's current state: the state fields' ghost layers are filled
 * first (mhd_sync of U and B faces), as the reference's checkpoint holds
 * them.  Synchronous. */
int mhd_batch_save_restart(mhd_batch *batch, int slot, const char *path);
/* Loads the state fields the file holds, fills their ghost layers and
 * prepares the solve at the file's time and step (*step, *time, may be
 * NULL), ready to step.  Synchronous. */
int mhd_batch_load_restart(mhd_batch *batch, int slot, const char *path, int32_t *step, double *time);
int mhd_save_restart(mhd_ctx *ctx, const char *path);
int mhd_load_restart(mhd_ctx *ctx, const char *path, int32_t *step, double *time);
/* The run-data file the reference writes beside each checkpoint
 * (IOModule::WriteRunDataFile -> RunData::WriteBinary,
 * include/6_io/RunData.h:96-149): step, time, the last step's dt, the
 * residual references (the Mercury solver: 13 values of 1.0,
 * Z4_Mercury/src/MercurySolver.cpp:29-30, src/6_io/IOModele_Basic.cpp:55),
 * residual_max (0) and the monitors (double and int32 values by key, written
 * in key order; the Mercury solver's are the run's performance figures,
 * src/6_io/RuntimeMonitor.cpp:28-55).  mhd_info gives step, time and dt.  The
 * reader returns step, time and dt.  Host-only. */
int mhd_rundata_write(const char *path, int32_t step, double time, double dt, int32_t nref,
                      const double *residual_ref, double residual_max, int32_t n_dmon, const char *const *dkeys,
                      const double *dvals, int32_t n_imon, const char *const *ikeys, const int32_t *ivals);
int mhd_rundata_read(const char *path, int32_t *step, double *time, double *dt);

/* ---- Checkpoint plot file ----
 * The Tecplot binary file (#!TDV112) the reference writes beside each
 * restart file (IOModule::WriteTecplotBinFile,
 * src/6_io/IOModule_Tecplot.cpp:749-1017) in the AllNode mode its Mercury
 * solver selects (Z4_Mercury/src/MercurySolver.cpp:49-86): per block one
 * ordered zone "Zone<b>_<name>" of (n + 1)^3 nodes; variables x, y, z and the
 * cell fields below averaged to the nodes, each node the |Jac|-weighted mean
 * of its eight cells (ghost cells included,
 * IOModule::EvalValue_CellToNode_), written as float after the per-variable
 * minimum and maximum.  Blocks without singular nodes (no averaging across
 * singular edges).  Host-only: the arrays are the ones mhd_download_field
 * returns (FieldBlock layout, (i, j, k, comp) order). */
#define MHD_TECPLOT_FIELDS 6 /* PV_H (5), PV_Na (5), B_cell (3), Bind_cell (3), Na (1), J_cell (3) */
typedef struct mhd_tecplot_image {
  int32_t n_blocks;
  const int32_t *cells;            /* 3 per block */
  const char *const *block_names;  /* per block */
  double time;                     /* solution time of the zones */
  const double *const *nodes;      /* per block: node x, y, z (3 components) over [0, n + 1) per axis */
  const double *const *jac;        /* per block: Jac over [-jac_ghost, n + jac_ghost) */
  int32_t jac_ghost;               /* >= 1 */
  const double *const *cell[MHD_TECPLOT_FIELDS]; /* per field, per block: over [-cell_ghost, n + cell_ghost) */
  int32_t cell_ghost;              /* >= 1 */
} mhd_tecplot_image;
int mhd_tecplot_write(const char *path, const mhd_tecplot_image *img);

#ifdef __cplusplus
}
#endif
#endif /* MERCURY_MHD_H */
