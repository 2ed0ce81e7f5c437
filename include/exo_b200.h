/*
 * exo_b200.h -- C ABI of the B200-native finite-volume step on the cubed sphere.
 *
 * This library re-implements, for NVIDIA B200 (sm_100a), the hot path of
 * ExoCubed's cubed-sphere dynamical core: Hydro::CalculateFluxes with WENO5
 * sweeps, the RiemannSolver hooks (Roe shallow water, LMARS, HLLC), the exo3
 * panel ghost-zone interpolation and panel-edge face-state exchange, the snap
 * hydrostatic pressure decomposition, the ImplicitSolver vertical correction
 * and the SSPRK(3,3) stage update.  All six panels of one atmosphere live on
 * one GPU.  Everything crosses this boundary as plain pointers and sizes.
 *
 * Array layout (host and device): one AthenaArray<Real>(n,k,j,i) per panel,
 * i (x1, radial) fastest, six panels back to back:
 *     a[((((p*nvar + n)*nc3 + k)*nc2 + j)*nc1 + i]
 * with nc1 = L + 2*EXO_NGHOST, nc2 = nc3 = N + 2*EXO_NGHOST, p = panel id - 1
 * (panel ids follow CubedSphere::FindBlockID, src/exo3/cs_find_block_id.cpp:11).
 *
 * Error convention: every entry point returns an int status, 0 on success;
 * no C++ exception crosses the boundary.  exo_last_error() gives the text of
 * the most recent failure on the calling thread.  A context is single-stream
 * and not thread safe: use one context per host thread.
 */
#ifndef EXO_B200_H_
#define EXO_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EXO_NGHOST 3
#define EXO_NPANEL 6

/* status codes */
enum {
  EXO_OK = 0,
  EXO_ERR_ARG = 1,        /* bad argument or configuration */
  EXO_ERR_SHAPE = 2,      /* array shape does not match the context */
  EXO_ERR_CUDA = 3,       /* CUDA runtime error (text in exo_last_error) */
  EXO_ERR_NONFINITE = 4,  /* state became invalid: rho<0, p<0 or NaN */
  EXO_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
  EXO_ERR_NOGPU = 6,      /* no CUDA device is usable */
  EXO_ERR_CAPACITY = 7    /* a request does not fit the slots or memory */
};

/* equation sets: the reference's EOS choice (src/snap/CMakeLists.txt:23) */
enum { EXO_EQN_SHALLOW_YZ = 0, EXO_EQN_IDEAL = 1 };

/* Riemann solvers: the reference's RSOLVER choice (src/snap/CMakeLists.txt:26) */
enum {
  EXO_RS_ROE_SHALLOW = 0,   /* src/snap/riemann/roe_shallow_yz.cpp   */
  EXO_RS_LMARS = 1,         /* src/snap/riemann/lmars.cpp            */
  EXO_RS_HLLC = 2,          /* src/snap/riemann/hllc_transform.cpp   */
  EXO_RS_LMARS_SHALLOW = 3  /* src/snap/riemann/lmars_shallow_yz.cpp */
};

/* arithmetic of the flux path */
enum {
  EXO_PREC_FP64 = 0,            /* everything in FP64 */
  EXO_PREC_MIXED = 1,           /* FP32 reconstruction, x2/x3 Riemann fluxes and
                                   their divergence; FP64 decomposition, x1
                                   (radial) fluxes and their divergence, implicit
                                   solve, state and RK accumulation */
  EXO_PREC_MIXED_F32_SOLVE = 2  /* EXO_PREC_MIXED with the implicit solve's blocks,
                                   their factorisation and its back-substitution
                                   factors in FP32 (faster solve, larger error;
                                   state and corrected update stay FP64) */
};

/* Coriolis source (a user explicit source of the reference's examples):
   W92: the lat-lon f-plane form of examples/2023-Chen-exo3/W92.cpp:48-70;
   3D:  CubedSphere::CalculateCoriolisForce3 (src/exo3/cubed_sphere.cpp:197-231),
        the full rotation vector on every panel, all three momenta */
enum { EXO_CORIOLIS_NONE = 0, EXO_CORIOLIS_W92 = 1, EXO_CORIOLIS_3D = 2 };
/* user forcing, added with the sources of each stage:
   HS94: examples/2023-Chen-exo3/hs94.cpp:59-155 -- Coriolis on the momenta in
         latitude-longitude, Rayleigh drag below sigmab and Newtonian cooling
         toward the Held-Suarez equilibrium temperature (uses omega, gamma,
         Rd and the hs_* parameters) */
enum { EXO_FORCING_NONE = 0, EXO_FORCING_HS94 = 1 };

typedef struct exo_config {
  int N;              /* cells along a panel edge (meshblock nx2 = nx3)          */
  int L;              /* radial levels (nx1)                                      */
  int eqn;            /* EXO_EQN_*                                                */
  int rsolver;        /* EXO_RS_*                                                 */
  int implicit_flag;  /* <hydro> implicit_flag bits: 1 = x1 (3x3 partial       */
                      /* correction), + 8 = full 5x5 correction                   */
  int precision;      /* EXO_PREC_*                                               */
  int coriolis;       /* EXO_CORIOLIS_*                                           */
  int forcing;        /* EXO_FORCING_*                                            */
  double x1min;       /* inner radius [m]                                         */
  double x1max;       /* outer radius [m]                                         */
  double gamma;       /* <hydro> gamma                                            */
  double Rd;          /* <thermodynamics> Rd [J/kg/K]                             */
  double grav;        /* <hydro> grav_acc1 (negative points down) [m/s^2]         */
  double cfl;         /* <time> cfl_number                                        */
  double omega;       /* planetary rotation rate for the Coriolis source [1/s]    */
  double reserved1;
  /* Held-Suarez forcing (hs94.inp <problem> and <thermodynamics> blocks) */
  double hs_p0;       /* p0: reference surface pressure [Pa]                      */
  double hs_Ts;       /* Ts: equatorial surface temperature [K]                   */
  double hs_dT;       /* dT: equator-to-pole temperature difference [K]           */
  double hs_dtheta;   /* dtheta: vertical potential temperature difference [K]    */
  double hs_Kf;       /* Kf: boundary-layer Rayleigh drag rate [1/day]            */
  double hs_Ka;       /* Ka: free-atmosphere Newtonian cooling rate [1/day]       */
  double hs_Ks;       /* Ks: surface Newtonian cooling rate [1/day]               */
  double hs_sigmab;   /* sigmab: top of the boundary layer, in p/p0               */
} exo_config;

typedef struct exo_ctx exo_ctx;

/* -------------------------------------------------------------- lifecycle */

/* Fill *cfg with the defaults of an equation set (C1 for shallow water, C2
   for the ideal gas).  Replaces the <mesh>/<hydro>/<time> blocks of an
   Athena++ input file (examples/2023-Chen-exo3/W92.inp, hs94.inp). */
int exo_config_default(exo_config* cfg, int eqn);

/* Create a context on the current CUDA device: geometry tables, panel
   interpolation tables and device state are allocated here, never later.
   Replaces Mesh/MeshBlock construction (src/mesh_setup.cpp:66) and the
   GnomonicEquiangle constructor (src/exo3/gnomonic_equiangle.cpp:24). */
int exo_create(const exo_config* cfg, exo_ctx** out);
void exo_destroy(exo_ctx* ctx);

/* Cell-centre geometry of a configuration, computed on the host (no GPU
   needed): lat, lon [6][N][N] in radians (CubedSphere::GetLatLon,
   src/exo3/cubed_sphere.cpp:78-91); uv_to_v23 [6][N][N][4] the map of a
   latitude-longitude vector (U east, V north) to the panel's contravariant
   components, V2 = c0*U + c1*V, V3 = c2*U + c3*V (CubedSphere::GetVyVz,
   cubed_sphere.cpp:149-162); x1v [L] the radial cell centres.  Any output
   pointer may be NULL. */
int exo_cell_geometry(const exo_config* cfg, double* lat, double* lon,
                      double* uv_to_v23, double* x1v);

/* Face coordinates of one panel (host, no GPU): x1f [L+7], x2f [N+7],
   x3f [N+7] in the reference's units (x1 radius in m; x2, x3 equiangular
   angles in rad) -- patches/27.coordinates.patch:21,40. */
int exo_mesh(const exo_config* cfg, int panel, double* x1f, double* x2f, double* x3f);

/* Number of variables and cell counts of one panel array. */
int exo_shape(const exo_ctx* ctx, int* nvar, int* nc3, int* nc2, int* nc1);

/* Text of the last error on this thread ("" if none). */
const char* exo_last_error(void);

/* ---------------------------------------------------------- state access */

/* Load an initial state given as primitive variables (interior cells are
   read, ghosts ignored) from host memory.  Runs what Mesh::Initialize does
   after ProblemGenerator: PrimitiveToConserved on the interior, the panel
   ghost exchange, ConservedToPrimitive, the physical x1 boundary and the
   first time step (patches/29.mesh.patch:19-86). */
int exo_set_primitive(exo_ctx* ctx, const double* w_host);

/* Copy the full conserved / primitive arrays (ghosts included) to host. */
int exo_get_conserved(exo_ctx* ctx, double* u_host);
int exo_get_primitive(exo_ctx* ctx, double* w_host);

/* Device pointers of the resident state (valid until exo_destroy). */
int exo_device_state(exo_ctx* ctx, double** u_dev, double** w_dev);

/* --------------------------------------------------------------- stepping */

/* Advance nsteps SSPRK(3,3) steps.  dt_fixed <= 0 selects the CFL time step
   of Hydro::NewBlockTimeStep (patches/21.new_blockdt.patch:23-35), recomputed
   on the device after every step; dt_fixed > 0 uses that step throughout.
   Replaces the main loop's DoTaskListOneStage calls (main.cpp.in:139-141). */
int exo_step(exo_ctx* ctx, int nsteps, double dt_fixed);

/* Current time step, simulated time and step count. */
int exo_get_dt(exo_ctx* ctx, double* dt);

/* One stage (0, 1, 2) of SSPRK(3,3) on the CFL time step: the reference's
   DoTaskListOneStage(stage) for the whole atmosphere (fluxes, update,
   implicit correction, boundaries, primitives); stage 2 also advances the
   time and computes the next step.  Three calls equal one exo_step. */
int exo_stage(exo_ctx* ctx, int stage);
/* The two ghost syncs of a stage and ConservedToPrimitive (PackData /
   unpack of the panel boundaries, cubed_sphere_utility.cpp:18-619, and the
   reflecting x1 ghosts): the primitives, ghosts included, from the current
   conserved state. */
int exo_boundary(exo_ctx* ctx);
/* ImplicitSolver::SolveImplicit3D(du, w, dt) (solve_implicit_3d.cpp:27-180,
   FullCorrection): du_host (six AthenaArray(NHYDRO, nc3, nc2, nc1) blocks,
   interior used) is corrected in place from the primitives w_host (ghosts
   used at the x1 boundaries) with time step dt.  It works in the context's
   own primitive and update arrays: load a state (exo_set_primitive) before
   stepping the context again. */
int exo_solve_implicit_3d(exo_ctx* ctx, double* du_host, const double* w_host, double dt);
/* Decomposition::ChangeToPerturbation(w, ...) (change_to_perturbation.cpp:
   39-157) on every radial column: w_host (six AthenaArray(NHYDRO, nc3, nc2,
   nc1) blocks, ghosts included; interior columns used) has the hydrostatic
   pressure (log mean of the face pressures integrated down from the top) and
   the isentropic reference density subtracted in place.  The context keeps
   the face pressures, the original pressure and density and each column's
   gamma and entropy for the restore (device memory allocated on the first
   call, freed by exo_destroy).  No-op without gravity, as in the reference. */
int exo_change_to_perturbation(exo_ctx* ctx, double* w_host);
/* Decomposition::RestoreFromPerturbation(w, wl, wr, k, j, il, iu)
   (:159-222) on every column: w_host gets its pressure and density back as
   they were before exo_change_to_perturbation; the x1 face states wl_host
   and wr_host (same layout as w; entry i is the face between cells i-1 and
   i, faces is..ie+1 used) get the face pressure and isentropic face density
   added back with the reference's positivity fallbacks.  Both calls work in
   the context's own device arrays: load a state before stepping again. */
int exo_restore_from_perturbation(exo_ctx* ctx, double* w_host, double* wl_host, double* wr_host);
int exo_get_time(exo_ctx* ctx, double* time, int64_t* ncycle);

/* Sticky device-side validity flag (MeshBlock::Impl::SetStateInvalid,
   src/snap/eos/ideal_moist_hydro.cpp:108,150): 1 if a density or pressure
   went negative or NaN since the last call; the flag is cleared.  Returns
   EXO_ERR_TIMEOUT (with *invalid set) once a kernel's bounded wait for its
   bulk copies into shared memory has given up; that kernel left the state
   of the columns it had not finished as the forward sweep left it. */
int exo_check_state(exo_ctx* ctx, int* invalid);

/* Block until the context's stream is idle. */
int exo_synchronize(exo_ctx* ctx);

/* The cudaStream_t every launch of this context goes to. */
int exo_get_stream(exo_ctx* ctx, void** stream);

/* ------------------------------------------------------------- profiling */

/* kernels of one stage, for exo_profile_read */
enum {
  EXO_K_FLUX_X1 = 0,    /* decomposition + WENO5 + Riemann, x1 (per column)  */
  EXO_K_FLUX_X23 = 1,   /* WENO5 + edge exchange + Riemann, x2/x3 (per face)  */
  EXO_K_UPDATE = 2,     /* RK average + divergence + sources (per cell)       */
  EXO_K_IMPLICIT = 3,   /* 5x5 block-tridiagonal vertical solve (per column)  */
  EXO_K_PRIM_GHOST = 4, /* ghost bands + ConservedToPrimitive + CFL (per cell) */
  EXO_K_OTHER = 5,      /* time-step bookkeeping                              */
  EXO_K_COUNT = 6
};

/* enable != 0 brackets every launch with CUDA events on the context's
   stream and clears the counters; 0 stops recording.  exo_profile_read
   synchronizes and returns the launches and the summed device time (ms) of
   one kernel since profiling was enabled. */
int exo_profile(exo_ctx* ctx, int enable);

/* Launch tiles: threads per block of each kernel, indexed by EXO_K_* (the
   EXO_K_OTHER slot is the last-stage AirParcel round trip of atmospheres
   without the implicit solver).  EXO_K_FLUX_X1 is the radial columns per
   block of the x1 kernel (1 to 8, its threads follow from L); the others
   take a multiple of 32 in [32, 512], EXO_K_IMPLICIT one of 32, 64, 128
   (radial columns per block); 0 keeps the current value.  The results do not depend on the tiles, only the speed
   does.  No counterpart in the reference (its CPU loops have no launch shape). */
#define EXO_TILE_COUNT 6
int exo_set_tiles(exo_ctx* ctx, const int* threads);
int exo_get_tiles(exo_ctx* ctx, int* threads);
int exo_profile_read(exo_ctx* ctx, int kernel, int64_t* launches, double* total_ms);

/* Kernel launches issued by this context since it was created. */
int exo_launch_count(exo_ctx* ctx, int64_t* launches);

/* ------------------------------------------------------ operator hooks */

/* Hydro::CalculateFluxes (patches/19.calculate_fluxes.patch:22-158) on the
   current primitive state; the three flux arrays stay on the device and can
   be copied out with exo_get_flux (dir = 0,1,2 for x1,x2,x3; layout as the
   state arrays, face index in place of cell index). */
int exo_calculate_fluxes(exo_ctx* ctx);
int exo_get_flux(exo_ctx* ctx, int dir, double* flux_host);

/* Hydro::RiemannSolver(k,j,il,iu,ivx,wl,wr,flx,dxw) over n faces stored as
   device arrays wl[NHYDRO][n], wr[NHYDRO][n] -> flx[NHYDRO][n] (all FP64).
   The face geometry enters as per-face arrays: cos_face/sin_face are the
   face metric (Face2Metric/Face3Metric, gnomonic_equiangle.cpp:494-569),
   cth_proj the covariant projection angle and cth_cell the cell-centred
   metric used by HLLC in x1 (hllc_transform.cpp:95-110); pass NULL where the
   solver does not use them.  Replaces src/snap/riemann/{roe_shallow_yz,
   lmars,hllc_transform,lmars_shallow_yz}.cpp. */
int exo_riemann(int rsolver, int eqn, int ivx, int n, double gamma,
                const double* wl, const double* wr, double* flx,
                const double* cos_face, const double* sin_face,
                const double* cth_proj, const double* cth_cell,
                void* stream);

/* ImplicitSolver::FullCorrection with SolveImplicit3D's velocity projection
   (src/snap/implicit/solve_implicit_3d.cpp:102-179, full_correction.cpp:32-165,
   forward_backward.hpp:15-126) over ncol independent radial columns, all
   arrays on the device:
     w       [ncol][5][L+6]  primitives incl. the 3+3 radial ghosts
     du      [ncol][5][L]    explicit update in, corrected update out
     colgeo  [ncol][4]       cos and sin of the cell metric, dx2f_ang, dx3f_ang
     x1f [L+7], x1v [L+6], dx1f [L+6]  radial faces, centres and widths
     scratch ncol*L*30 doubles of caller-owned device memory
   Reflecting radial boundaries at both ends; dt is the stage's beta*dt. */
int exo_implicit_columns(int ncol, int L, const double* w, double* du,
                         const double* colgeo, const double* x1f, const double* x1v,
                         const double* dx1f, double dt, double gamma, double grav,
                         double* scratch, void* stream);

/* ImplicitSolver::PartialCorrection with SolveImplicit3D's velocity
   projection (src/snap/implicit/solve_implicit_3d.cpp:102-179,
   partial_correction.cpp:26-173, forward_backward.hpp:15-126) over ncol
   independent radial columns: the 3x3 block-tridiagonal system of
   (rho, x1 momentum, energy).  Arguments as for exo_implicit_columns; the
   x2 and x3 momentum rows of du are left as they came in. */
int exo_partial_correction_columns(int ncol, int L, const double* w, double* du,
                                   const double* colgeo, const double* x1f,
                                   const double* x1v, const double* dx1f, double dt,
                                   double gamma, double grav, double* scratch,
                                   void* stream);

/* Allocation-free form of exo_implicit_columns.  This entry point has no
   counterpart in the reference: it exists for callers that cannot allocate
   device memory at the moment they advance the solution -- a host
   application whose memory pool reserved the GPU up front (cudaMalloc would
   fail or fragment it), a time-stepping or serving loop that must not stall
   on the device-wide synchronization cudaMalloc/cudaFree can cause, or a
   caller held to a fixed memory budget.  The caller passes inputs and
   outputs exactly as for exo_implicit_columns; the 30 scratch doubles per
   column level live in one fixed device array of EXO_NOALLOC_SCRATCH_DOUBLES
   (8 MiB) that the library holds on every GPU it is loaded on, so
   ncol * L must not exceed EXO_NOALLOC_SCRATCH_DOUBLES / 30 = 34952 (e.g.
   546 columns of 64 levels); larger batches return EXO_ERR_CAPACITY.
   The first call on each device looks up the array's device address (with
   that device current); make that first call before any stream capture.
   All calls share the one array and nothing in it needs to start at zero
   (every word a column reads was written earlier in the same call), but
   calls that overlap on the GPU -- other streams, other threads -- race on
   it: issue them in order on one stream. */
#define EXO_NOALLOC_SCRATCH_DOUBLES 1048576
int exo_implicit_columns_noalloc(int ncol, int L, const double* w, double* du,
                                 const double* colgeo, const double* x1f,
                                 const double* x1v, const double* dx1f, double dt,
                                 double gamma, double grav, void* stream);

/* interp_weno5 on device: out[m] = weno5(a[m],b[m],c[m],d[m],e[m]), the
   face value between the 2nd and 3rd argument (tests/test_weno.cpp:20-29). */
int exo_weno5(int n, const double* a, const double* b, const double* c,
              const double* d, const double* e, double* out, void* stream);

/* out[m] = 1/x[m] on device as the implicit solve's FP64 blocks of the given
   precision compute it: an IEEE division in the FP64 build, a reciprocal
   refined by Newton's method in the mixed build (within an ulp or two).  A
   self-test of that arithmetic; x and out are device arrays of n doubles. */
int exo_reciprocal(int precision, int n, const double* x, double* out, void* stream);

/* ------------------------------------------------- panel-exchange hooks */

/* CubedSphereUtility::PackData (src/exo3/cubed_sphere_utility.hpp:10-12,
   cubed_sphere_utility.cpp:370-619) for a context's panel: src is one
   panel's array (NHYDRO, N+6, N+6, L+6) on the device, buf a device buffer
   written from buf[*offset] on, *offset advanced by the values written.
   Across a panel edge (ox1 = 0, exactly one of ox2, ox3 non-zero; the
   ranges the G-wide interior band LoadBoundaryBufferSameLevel passes, every
   variable) the band is interpolated onto the neighbour's ghost cells and
   its vectors rotated into the neighbour's basis (InteprolateX2/X3), in the
   order PackDataR0..R3 give, so the neighbour unpacks it in plain
   (n, k, j, i) order; corners and radial neighbours are copied as
   PackDataR0 does.  EXO_ERR_SHAPE for other ranges.  stream NULL: the
   context's stream.  The reference's bound_lim > 0 (several blocks per
   panel) has no counterpart: a context is one block per panel. */
int exo_panel_pack(exo_ctx* ctx, const double* src, double* buf, int sn, int en, int si,
                   int ei, int sj, int ej, int sk, int ek, int* offset, int ox1, int ox2,
                   int ox3, int panel, void* stream);

/* CubedSphere::SaveLR3DValues / LoadLR3DValues (src/exo3/cubed_sphere.hpp:
   47-50, cubed_sphere.cpp:267-287): store and read back one row of x2
   (direction 2) or x3 (direction 3) face states, L_row and R_row
   [NHYDRO][L+6] (host or device memory), faces il..iu of row (k, j) of a
   panel, in the context's face-state stores (device memory allocated on the
   first call, four arrays of the state's size).  exo_lr3d_arrays returns
   those stores (device pointers, the state's (panel, n, k, j, i) layout) for
   callers that fill or read them whole. */
int exo_save_lr3d(exo_ctx* ctx, const double* L_row, const double* R_row, int direction,
                  int panel, int k, int j, int il, int iu, void* stream);
int exo_load_lr3d(exo_ctx* ctx, double* L_row, double* R_row, int direction, int panel,
                  int k, int j, int il, int iu, void* stream);
int exo_lr3d_arrays(exo_ctx* ctx, double** L2, double** R2, double** L3, double** R3);
/* CubedSphere::SynchronizeFluxesSend / Recv / Wait (cubed_sphere.cpp:
   289-688) on the stores: at every panel-edge face (faces is-1..ie+1) the
   neighbour's interior-side state, rotated into this panel's basis, becomes
   the outer state (L at the Up/Left edges, R at Down/Right).  One kernel on
   the device instead of MPI messages. */
int exo_synchronize_faces(exo_ctx* ctx, void* stream);

/* ---------------------------------------------- equation-of-state hooks */

/* EquationOfState::ConservedToPrimitive / PrimitiveToConserved
   (src/snap/eos/ideal_moist_hydro.cpp:77-196, shallow_yz_hydro.cpp:42-107)
   on cells [il,iu] x [jl,ju] x [kl,ku] of every panel; u and w are device
   arrays in the context's (panel, n, k, j, i) layout, ghosts included.
   Covariant momenta become contravariant velocities with the cell metric as
   in the reference; a negative or non-finite density or pressure sets the
   sticky flag exo_check_state reads (SetStateInvalid). */
int exo_conserved_to_primitive(exo_ctx* ctx, const double* u, double* w, int il, int iu,
                               int jl, int ju, int kl, int ku, void* stream);
int exo_primitive_to_conserved(exo_ctx* ctx, const double* w, double* u, int il, int iu,
                               int jl, int ju, int kl, int ku, void* stream);
/* EquationOfState::SoundSpeed (ideal_moist_hydro.cpp:226-238,
   shallow_yz_hydro.cpp:103-107) of n cells: prim [NHYDRO][n] -> cs [n],
   device arrays. */
int exo_sound_speed(exo_ctx* ctx, int n, const double* prim, double* cs, void* stream);

/* ---------------------------------------------------------- array views */

/* A strided 4-D view of one panel's array, AthenaArray(n, k, j, i) order:
   element (n,k,j,i) at data + n*stride[0] + k*stride[1] + j*stride[2] +
   i*stride[3] (strides in elements, any sign).  device < 0: host memory;
   otherwise the device memory of that CUDA device (the context's). */
#define EXO_DTYPE_F64 0
typedef struct exo_array_view {
  void* data;
  int dtype;              /* EXO_DTYPE_F64 */
  int nx4, nx3, nx2, nx1; /* NHYDRO, N+6, N+6, L+6 */
  int64_t stride[4];
  int device;
} exo_array_view;

/* The whole-array entry points on six panel views (views[p] = panel p), the
   reference's one AthenaArray per MeshBlock: exo_set_primitive,
   exo_get_primitive, exo_get_conserved and exo_solve_implicit_3d (du in and
   out, w in) with their arrays gathered from and scattered to the views. */
int exo_set_primitive_views(exo_ctx* ctx, const exo_array_view* w);
int exo_get_primitive_views(exo_ctx* ctx, const exo_array_view* w);
int exo_get_conserved_views(exo_ctx* ctx, const exo_array_view* u);
int exo_solve_implicit_3d_views(exo_ctx* ctx, const exo_array_view* du,
                                const exo_array_view* w, double dt);

/* ------------------------------------------------------------- ensembles */

/* A batch of independent atmospheres of uneven size (different N, L, gas,
   gravity, solver) advanced together: every kernel of a step is launched
   once for all members and the step is one CUDA graph.  This is the
   forward-model workload of the reference's MCMC inversion
   (src/inversion/profile_inversion.cpp:112-120), which the reference runs as
   one atmosphere per process.  Members are admitted against a device-memory
   budget (bytes) and a slot capacity; their memory comes from the
   ensemble's own stream-ordered pool.  All members share one precision. */
typedef struct exo_ensemble exo_ensemble;

int exo_ensemble_create(int precision, int capacity, size_t budget_bytes,
                        exo_ensemble** out);
void exo_ensemble_destroy(exo_ensemble* ens);

/* Device bytes one member of this configuration holds (state, scratch,
   tables); host only. */
int exo_ensemble_footprint(const exo_config* cfg, size_t* bytes);

/* Admit a member with the primitive initial state w_host (layout as for
   exo_set_primitive).  EXO_ERR_CAPACITY if no slot is free or its footprint
   does not fit the remaining budget.  *slot receives its slot index. */
int exo_ensemble_add(exo_ensemble* ens, const exo_config* cfg, const double* w_host,
                     int* slot);
int exo_ensemble_remove(exo_ensemble* ens, int slot);

/* Advance every member nsteps SSPRK(3,3) steps, each with its own CFL time
   step (asynchronous; exo_ensemble_synchronize waits). */
int exo_ensemble_step(exo_ensemble* ens, int nsteps);
int exo_ensemble_synchronize(exo_ensemble* ens);

int exo_ensemble_get_conserved(exo_ensemble* ens, int slot, double* u_host);
int exo_ensemble_get_primitive(exo_ensemble* ens, int slot, double* w_host);
int exo_ensemble_member_time(exo_ensemble* ens, int slot, double* time, double* dt,
                             int64_t* ncycle);
/* Launch tiles of the batched step (as exo_set_tiles); the next
   exo_ensemble_step re-captures its graph with them. */
int exo_ensemble_set_tiles(exo_ensemble* ens, const int* threads);
int exo_ensemble_get_tiles(exo_ensemble* ens, int* threads);
/* MeshBlock::Impl::IsStateValid for one member: the sticky device flag set
   when a cell's density or pressure turned non-positive or NaN, cleared on
   read (as exo_check_state). */
int exo_ensemble_check_state(exo_ensemble* ens, int slot, int* invalid);
/* Members admitted, device bytes held by them, kernel launches issued. */
int exo_ensemble_stats(exo_ensemble* ens, int* members, size_t* bytes_in_use,
                       int64_t* launches);
int exo_ensemble_get_stream(exo_ensemble* ens, void** stream);

/* ------------------------------------------------------ redo of a step */

/* The main loop's redo of failed steps (main.cpp.in:126-157,
   src/mesh_redo.cpp:12-46): with max_redo > 0 every exo_step step first
   keeps a device copy of u, w (with the FP32 primitive copy of the mixed
   builds) and the clock; a step that leaves the state
   invalid (rho or p negative or not finite, exo_check_state) is taken again
   from that copy with half the time step (half the fixed dt when one is
   given), as often as needed.  As in the reference the budget counts redos
   over the whole run and `attempts++ > max_redo` ends it: the step returns
   EXO_ERR_NONFINITE with the kept state back in place and its dt halved.
   A step that starts from an invalid state returns EXO_ERR_NONFINITE at
   once.  Each step then waits for the device once (the flag read); the
   default 0, the reference's, keeps steps asynchronous.  The first call with
   max_redo > 0 allocates the copy (2 x the state, 2.5 x in the mixed
   builds). */
int exo_set_max_redo(exo_ctx* ctx, int max_redo);
/* Redos taken so far. */
int exo_redo_count(exo_ctx* ctx, int64_t* redos);

/* ----------------------------------------------------------- checkpoints */

/* A checkpoint image holds what a run needs to continue exactly where it
   stopped: the configuration, the clock (time, steps taken, the dt of the
   next step) and the conserved and primitive arrays with their ghosts.  It
   replaces the hydro part of an Athena++ restart file (src/mesh_setup.cpp:
   25-97, written by <output> file_type = rst in hs94.inp) and of the
   in-memory copy MeshBlock::Impl::SaveAllStates / LoadAllStates keeps
   (src/impl.cpp:306-332).  A run resumed from an image takes, step for step,
   the bits the uninterrupted run takes.
   Layout: exo_checkpoint_header (512 bytes), then u, then w, each
   header.values doubles in the context's (panel, variable, k, j, i) order,
   in the byte order of the machine that wrote it. */
#define EXO_CHECKPOINT_VERSION 1
typedef struct exo_checkpoint_header {
  char magic[8];          /* "EXOCKPT1" (not NUL-terminated)                  */
  uint32_t version;       /* EXO_CHECKPOINT_VERSION                           */
  uint32_t header_bytes;  /* sizeof(exo_checkpoint_header) = 512              */
  uint64_t values;        /* doubles in each of u and w: 6*nvar*nc3*nc2*nc1   */
  double time;            /* simulated time                                   */
  double dt;              /* the step the run takes next                      */
  int64_t ncycle;         /* steps taken                                      */
  int32_t invalid;        /* sticky invalid-state flag at the time of writing */
  int32_t reserved;
  exo_config cfg;         /* the configuration the state belongs to           */
  uint8_t pad[512 - 56 - sizeof(exo_config)];
} exo_checkpoint_header;

/* Bytes of a checkpoint image of this context (header + u + w). */
int exo_checkpoint_bytes(const exo_ctx* ctx, size_t* bytes);
/* Write the context's image into image[0, bytes): waits for the context's
   queued work.  EXO_ERR_SHAPE if bytes is smaller than exo_checkpoint_bytes. */
int exo_checkpoint_save(exo_ctx* ctx, void* image, size_t bytes);
/* Continue from an image: its configuration must equal the context's in
   every field except precision (a run may resume in the other build);
   EXO_ERR_ARG for a foreign or damaged image or another configuration. */
int exo_checkpoint_load(exo_ctx* ctx, const void* image, size_t bytes);
/* The same for one member of an ensemble, and admission of a new member
   from an image (in the ensemble's precision), which then continues the run
   that wrote it. */
int exo_ensemble_checkpoint_bytes(exo_ensemble* ens, int slot, size_t* bytes);
int exo_ensemble_checkpoint_save(exo_ensemble* ens, int slot, void* image, size_t bytes);
int exo_ensemble_add_checkpoint(exo_ensemble* ens, const void* image, size_t bytes, int* slot);

/* --------------------------------------------------------- measurement */

/* Arithmetic ceiling of the current device: the rate of fused multiply-adds
   (2 flops each) that a kernel of independent FMA chains in FP64 (fp64 = 1)
   or FP32 (fp64 = 0) reaches on all SMs, timed with CUDA events on the
   default stream after one warm-up launch; *flops_per_s receives the best of
   `repeats` launches.  No counterpart in the reference (its only instrument
   is the zone-cycles print of src/mesh_destroy.cpp:43-63): it gives the
   roofline of the step's FP64-issue-bound kernels a measured denominator. */
int exo_measure_fma_peak(int fp64, int repeats, double* flops_per_s);

/* Failure detection without a fault: one warp of a one-block kernel waits
   on an mbarrier phase that nothing will complete, through the bounded
   wait the library's kernels use for their bulk copies; it gives up after
   0.1 s of wall time and returns.  *gave_up receives 1 (the wait ran out and
   the kernel ended normally), *waited_ms how long it waited.  No
   counterpart in the reference (its waits are MPI calls). */
int exo_check_bounded_wait(int* gave_up, double* waited_ms);

#ifdef __cplusplus
}
#endif

#endif /* EXO_B200_H_ */
