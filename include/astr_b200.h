/*
 * astr_b200.h — C ABI of the B200 (sm_100a) implementation of ASTR's per-step RHS hot path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an int status
 * (ASTR_OK = 0, negative on error, never aborts) and records a message readable through
 * astr_last_error(). A call on a context (or on a scheme, state, ensemble or adjoint made from
 * one) runs on the context's device and restores the caller's current device before returning.
 * Arrays crossing the boundary are Fortran-ordered (first index fastest) with explicit lower
 * bounds, so a Fortran caller passes c_loc(f(lb0,lb1,lb2)) together with shape(f) and lbound(f). `where` says whether a pointer is host (ASTR_HOST) or device
 * (ASTR_DEVICE) memory; host pointers are only borrowed for the duration of the call.
 *
 * Reference interfaces replaced (paths inside Perrbit/astr_gpu):
 *   astr_fd_scheme_create   fd_scheme_initiate(asolver,scheme,ntype,dim,dir)  src/derivative.F90:63
 *   astr_filter_create      filter_coefficient_cal(alfa,beter_halo,beter_bouond) src/filter.F90:299
 *                           + compact_filter_initiate(afilter,ntype,dim,note)  src/filter.F90:31
 *   astr_scheme_ac          compact_scheme%ac (tridiagonal_thomas_proprocess)  src/commtype.F90:13-23,
 *                                                                              src/commfunc.F90:752
 *   astr_deriv_lines        df = fds%central(asolver,f,dim) over every line    src/derivative.F90:22-41,171
 *   astr_filter_lines       ff = compact_filter(afilter,f,dim[,note])          src/filter.F90:112
 *   astr_flux_create        compact_flux_initiate(asolver,scheme,ntype,dim,wind) src/flux.F90:32-112
 *   astr_flux_lines         fh = flux_compact(asolver,f,dim), fh(-1:dim)       src/flux.F90:125-150
 *   astr_flux_diff_lines    qrhs += Fh(i) - Fh(i-1) of the compact flux         src/solver.F90:1509-1513,
 *                                                                              src/test.F90:755-765
 *   astr_state_*            the module arrays q/rho/vel/prs/tmp of commarray  miniapps/tgv_solver_3d/
 *                                                                              tgvsolver.F90:1-40
 *   astr_state_init_tgv     flowfield_init                                    tgvsolver.F90:172-234
 *   astr_cfl_dt             cflcal (spectral radius sum, dt held fixed)        src/commcal.F90:27-87
 *   astr_rhs                rhscal (gradcal, convection, -qrhs, diffusion)      tgvsolver.F90:962-992
 *   astr_rk3_step           rk3 x nsteps (SSP-RK3, filter after each stage)     tgvsolver.F90:994-1082,
 *                                                                              steploop :944-960
 *   astr_history            stacal rows (nstep, time, tke, enstrophy) + dissipation
 *                                                                              tgvsolver.F90:893-942,
 *                                                                              src/statistic.F90:993-1040
 *   astr_rk3_step_host      one call of rk3 with the state in host memory: upload, nsteps, download
 *   astr_full_*             time_integration_rk / rhscal of the full solver     src/mainloop.F90:298-476,
 *                                                                              src/solver.F90:184-283
 *   astr_h5io_init/_end     h5io_init(filename,mode) / h5io_end                src/hdf5io.F90:86-163
 *   astr_h5write_r8/_i4     h5write (h5wa3d_r8_struct, h5w_int4, h5srite)      src/hdf5io.F90:684-808,
 *                                                                              :1015-1100
 *   astr_h5read_r8/_i4      h5read (h5ra3d_r8_struct/_stream, h5r_int4)        src/hdf5io.F90:175-452
 *   astr_*_write_flowfield  writeflfed's flow field (write_io_tree + h5srite)  src/readwrite.F90:1720-1980
 *   astr_*_read_flowfield   readcheckpoint's flow field + updateq              src/readwrite.F90:1378-1528,
 *                                                                              src/fludyna.F90:254-300
 */
#ifndef ASTR_B200_H
#define ASTR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ASTR_OK = 0,
  ASTR_ERR_ARG = -1,         /* bad argument (null pointer, size, unsupported ntype/scheme) */
  ASTR_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  ASTR_ERR_STATE = -3,       /* device-side invalid state (non-finite or non-positive density) */
  ASTR_ERR_UNSUPPORTED = -4, /* size outside what the compiled kernels cover */
  ASTR_ERR_NOMEM = -5        /* device allocation failed */
};
enum { ASTR_HOST = 0, ASTR_DEVICE = 1 };

typedef struct astr_ctx astr_ctx;
typedef struct astr_scheme astr_scheme;
typedef struct astr_state astr_state;

/* Flow and scheme parameters of one periodic box (commvar of the reference). */
typedef struct {
  int im, jm, km;          /* nodes 0..im etc.; im = N means N^3 unique points, (N+1)^3 stored */
  double mach, reynolds, prandtl, gamma;
  double ref_tem;          /* 273.15 */
  double sutherland;       /* Sutherland constant in kelvin: 110.4 (miniapp) or 110.3 (full solver) */
  double alfa_filter;      /* 0.49 */
  double beta_halo;        /* 1.11 */
  double beta_bound;       /* 1.09 (miniapp) or 0.98 (full solver) */
  int filter_on;           /* apply filterq after every RK stage */
  int ntype[3];            /* per direction: 0 or 3 periodic; 1, 2, 4 physical ends (full-solver
                              mode only: fd_scheme_initiate's ntype, compact boundary closures) */
  double twall;            /* temperature of the isothermal no-slip walls at physical ends (bctype 41) */
  int conschm;             /* convection scheme of the full-solver mode: 0 or 643 the central compact
                              scheme (convrsdcal6); 543 the upwind compact interface flux with
                              Steger-Warming splitting and the MP limiter (convrsdcmp, no
                              characteristic decomposition). The miniapp step is central only. */
  double bfacmpld;         /* b factor of the upwind compact flux (bfacmpld of the input) */
  int lchardecomp;         /* conschm 543: limit in characteristic variables (chardecomp, Roe
                              averages) with the Ducros shock sensor (ducrossensor); periodic
                              directions only */
  double shkcrt;           /* the Ducros sensor's threshold (shkcrt of the input) */
} astr_params;

/* ---- context ------------------------------------------------------------------------ */
int astr_init(int device, astr_ctx** ctx);
int astr_destroy(astr_ctx* ctx);
const char* astr_last_error(astr_ctx* ctx);
/* Use the caller's CUDA stream (cudaStream_t) for all later work of this context. */
int astr_set_stream(astr_ctx* ctx, void* cuda_stream);
int astr_synchronize(astr_ctx* ctx);

/* ---- schemes (line operators) ----------------------------------------------------- */
/* scheme: "643c" (6th-order compact) or "643e" (explicit 6th-order, diff6ec). ntype 1..4 as in
 * fd_scheme_initiate: 1 boundary at i=0, 2 boundary at i=dim, 3 inner/periodic, 4 both. */
int astr_fd_scheme_create(astr_ctx* ctx, const char scheme[4], int ntype, int dim, astr_scheme** out);
/* compact 10th-order filter with LHS coefficient alpha_f; boundary_no_filter selects the
 * note='boundary_no_filter' variant of compact_filter_initiate. */
int astr_filter_create(astr_ctx* ctx, int ntype, int dim, double alpha_f, double beta_halo,
                       double beta_bound, int boundary_no_filter, astr_scheme** out);
int astr_scheme_destroy(astr_scheme* s);
/* Pre-factored Thomas table ac(3, first:last): ac[3*r + c], r = 0..last-first. */
int astr_scheme_ac(const astr_scheme* s, double* ac, int* first_node, int* last_node);

/* ---- line-level operators --------------------------------------------------------- */
/* Apply the scheme along dir (0,1,2) to every line of f: for each index pair of the output's
 * other two axes and t = 0..dim along dir,
 *     df(t) = scale * fds%central(asolver, f(-hm:dim+hm), dim)(t).
 * f(f_lb : f_lb+f_shape-1, ..., 1:nfields) must hold the line's halo nodes -5..dim+5 along dir
 * when the scheme reads them (ntype 1..3); df's range along dir must cover 0..dim and its other
 * axes must lie inside f's. */
int astr_deriv_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f,
                     const int64_t f_shape[3], const int64_t f_lbound[3], double* df,
                     const int64_t df_shape[3], const int64_t df_lbound[3], int nfields,
                     double scale, int where);
int astr_filter_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f,
                      const int64_t f_shape[3], const int64_t f_lbound[3], double* ff,
                      const int64_t ff_shape[3], const int64_t ff_lbound[3], int nfields, int where);

/* ---- compact interface flux (upwind-biased compact scheme) ------------------------- */
/* The '543' scheme of compact_flux_initiate: scheme must be 543; wind '+' (upwind-biased, the
 * reference's flux_uw_*) or '-' (downwind-biased, flux_dw_*); bfac is the MP-LD b factor
 * (bfacmpld of the reference's input). ntype 1..4 as for the derivative. */
int astr_flux_create(astr_ctx* ctx, int scheme, int ntype, int dim, char wind, double bfac,
                     astr_scheme** out);
/* Interface values fh(-1..dim) of every line along dir (interface i lies between nodes i and
 * i+1): f as for astr_deriv_lines (nodes -5..dim+5 where the scheme reads them), fh's range
 * along dir must cover -1..dim. */
int astr_flux_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f,
                    const int64_t f_shape[3], const int64_t f_lbound[3], double* fh,
                    const int64_t fh_shape[3], const int64_t fh_lbound[3], int nfields, int where);
/* The flux-form derivative: df(n) = scale * (fh(n) - fh(n-1)) at nodes 0..dim, fh as above
 * (never stored); accumulate != 0 adds it to df (device arrays only). */
int astr_flux_diff_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f,
                         const int64_t f_shape[3], const int64_t f_lbound[3], double* df,
                         const int64_t df_shape[3], const int64_t df_lbound[3], int nfields,
                         double scale, int accumulate, int where);

/* ---- solver state and the RK3 step ------------------------------------------------ */
int astr_state_create(astr_ctx* ctx, const astr_params* p, astr_state** out);
int astr_state_destroy(astr_state* st);
int astr_state_init_tgv(astr_state* st);
/* Conserved variables q(lb.., 1:5) on nodes 0..im x 0..jm x 0..km (any halo in the caller's
 * array is ignored on upload and left untouched on download). A host array of exactly those nodes
 * moves as one contiguous copy; when it is ordinary (pageable) memory of 32 MB or more, the copy
 * goes through the library's pinned staging memory (128 MB, kept once allocated, shared with the
 * checkpoint calls) with up to 8 host threads, and a pageable array with halos moves whole (only
 * its node rows are written back). The same holds for astr_rk3_step_host and the full solver's
 * upload and download. */
int astr_state_upload(astr_state* st, const double* q, const int64_t shape[3], const int64_t lbound[3], int where);
int astr_state_download(astr_state* st, double* q, const int64_t shape[3], const int64_t lbound[3], int where);
/* dt such that cflcal's CFL equals `cfl` on the current state. */
int astr_cfl_dt(astr_state* st, double cfl, double* dt);
/* One rhscal of the current state into qrhs(lb.., 1:5) on nodes 0..im etc. */
int astr_rhs(astr_state* st, double* qrhs, const int64_t shape[3], const int64_t lbound[3], int where);
int astr_rk3_step(astr_state* st, double dt, int nsteps);
/* The same, with the state in host memory for the duration of the call. */
int astr_rk3_step_host(astr_state* st, double* q, const int64_t shape[3], const int64_t lbound[3],
                       double dt, int nsteps, double diag_out[3]);
/* stacal rows written so far: (nstep, time, tke, enstrophy, dissipation), 5 doubles per row. */
int astr_history(astr_state* st, double* rows, int maxrows, int* nrows);
/* tke, enstrophy, dissipation of the current state (one gradient evaluation). */
int astr_diagnostics(astr_state* st, double out[3]);
/* Capture each RK3 step as one CUDA graph (default on). */
int astr_state_use_graph(astr_state* st, int on);
/* Apply the filter along y owed by each RK3 stage as its own pass (on) or fused into the first
 * gradient pass (off, the default); the autotuner times both at the first step and keeps the
 * faster unless this call (which turns autotuning off) or a pinned launch shape came first.
 * The two differ by rounding only (filterq, tgvsolver.F90:791-883). */
int astr_state_split_filter(astr_state* st, int on);
/* Per-pass autotuning of the launch shape (rows per lane, warps per line, lines per CTA) at the
 * first RK3 step of a state, on scratch copies of the live fields (default on above 100^3 nodes). */
int astr_state_autotune(astr_state* st, int on);
/* Launch shape of each pass A, B, C, A', B', filter-C, filter-A as (S, WPL, TI, LP, LPW, FPS):
 * 42 ints. */
int astr_state_launch_shapes(astr_state* st, int shapes[42]);
/* Pin pass `pass` (0..6 in the order above) to S rows per lane, WPL warps per line, TI lines per
 * CTA (a compiled layout whose 32*WPL*S rows cover the pass's line systems; TI a power of 2 with
 * (TI/LPW)*WPL*32 <= 512 threads, and TI/LPW <= 15 when WPL > 1) and
 * LPW lines per warp group (1; or a divisor of TI for the y/z passes A', B' and filter-A, whose
 * warps then loop over LPW lines of the tile) and FPS fields per step (5: all fields of the pass
 * at once; or 1 for A', B' and the filter passes, which then stream their independent fields one
 * at a time; LPW 2 needs FPS 1). */
int astr_state_set_launch_shape(astr_state* st, int pass, int S, int WPL, int TI, int LPW, int FPS);
/* Instrumentation (no counterpart in the reference): run `nsteps` RK3 steps eagerly with CUDA
 * events around every pass launch on the context stream and return the mean device time of
 * one launch of each pass, ms[0..7] = A, B, C, A', B', filter-C, diagnostics reduce, filter-A. */
int astr_pass_timings(astr_state* st, double dt, int nsteps, double ms[8]);

/* ---- batched ensemble ---------------------------------------------------------------- */
/* Several independent boxes (each an astr_state of the same context, sizes may differ)
 * advanced together: every pass of an RK3 stage is one launch per group of boxes sharing a
 * solve layout, and each ensemble step is one CUDA graph. No counterpart in the reference
 * (ASTR runs one block per MPI rank); the per-box results equal astr_rk3_step's. */
typedef struct astr_ensemble astr_ensemble;
int astr_ensemble_create(astr_ctx* ctx, astr_state* const* boxes, int nbox, astr_ensemble** out);
int astr_ensemble_destroy(astr_ensemble* e);
/* nsteps RK3 steps of every box; dt[b] is box b's time step. History rows go to each box. */
int astr_ensemble_step(astr_ensemble* e, const double* dt, int nsteps);

/* ---- discrete adjoint ---------------------------------------------------------------- */
/* Gradient of the final volume-averaged kinetic energy J = sum_{nodes 1..N} |rho u|^2/(2 rho) /
 * (im jm km) of nsteps RK3 steps (compact scheme, filter) with respect to the initial conserved
 * variables, by the discrete adjoint of the step: transposed compact solves and stencils,
 * pointwise vector-Jacobian products of the fluxes, reverse SSP-RK3 with a checkpoint every
 * `checkpoint_every` steps. No counterpart in the reference (ASTR has no adjoint); the forward
 * steps are the reference's rk3/rhscal (tgvsolver.F90:962-1082). Periodic boxes only. */
typedef struct astr_adjoint astr_adjoint;
int astr_adjoint_create(astr_state* st, int checkpoint_every, astr_adjoint** out);
int astr_adjoint_destroy(astr_adjoint* adj);
/* Advance the state nsteps steps from its current q, keeping checkpoints; *J = the objective. */
int astr_adjoint_forward(astr_adjoint* adj, double dt, int nsteps, double* J);
/* dJ/dq(step 0) into grad (5 fields of nodes 0..N, Fortran order, host or device). */
int astr_adjoint_backward(astr_adjoint* adj, double* grad, const int64_t shape[3], const int64_t lbound[3], int where);
/* lam_out = (d step/d q)^T lam_in for one step of size dt at the state's q (state unchanged). */
int astr_step_vjp(astr_adjoint* adj, double dt, const double* lam_in, double* lam_out, const int64_t shape[3],
                  const int64_t lbound[3], int where);
/* out = scale * L^T g along dir for a periodic scheme L (device arrays of dims, nodes 0..N along dir). */
int astr_scheme_apply_transpose(astr_ctx* ctx, astr_scheme* s, int dir, const double* g, const int64_t dims[3],
                                double* out, int nfields, double scale);

/* ---- full-solver time integration ------------------------------------------------ */
/* The full solver's rk3 stage (time_integration_rk, src/mainloop.F90:298-476) on a periodic box
 * of one rank with a uniform grid, on the reference's array layout (nodes -5..N+5 on every axis,
 * halos stored): filterq first (src/comsolver.F90:514-632), qswap (src/parallel.F90:4877-5060:
 * periodic halo copy, average of nodes 0 and N, primitives recomputed on the boundary planes and
 * halos only, so interior primitives stay those of the unfiltered state), rhscal in its metric
 * form (src/solver.F90:184-283, 2174-2874; src/comsolver.F90:244-497), the update of q*jacob
 * (src/mainloop.F90:426-446) and updatefvar (src/fludyna.F90:191-242). p->sutherland is 110.3 in
 * the full solver (src/solver.F90:121-122). History rows as astr_history (stage 1 of each step).
 * Directions with p->ntype 1, 2 or 4 take the compact boundary closures (derivative.F90:230-281,
 * filter.F90:176-249, with p->beta_bound) and isothermal no-slip walls at their physical ends
 * (boucon's noslip, src/bc.F90:6281-6595, applied after filterq at every stage). The miniapp step
 * (astr_state_*) is periodic only and rejects other ntypes. */
typedef struct astr_full astr_full;
int astr_full_create(astr_ctx* ctx, const astr_params* p, astr_full** out);
int astr_full_destroy(astr_full* fs);
/* Conserved variables on nodes 0..N of the caller's Fortran array q(lb.., 1:5); the primitives are
 * computed from them (updatefvar). Halo entries of the caller's array are ignored on upload and
 * left untouched on download. */
int astr_full_upload(astr_full* fs, const double* q, const int64_t shape[3], const int64_t lbound[3], int where);
int astr_full_download(astr_full* fs, double* q, const int64_t shape[3], const int64_t lbound[3], int where);
/* nsteps calls of time_integration_rk (rk3) with time step dt. */
int astr_full_step(astr_full* fs, double dt, int nsteps);
/* One stage's filterq + qswap + rhscal of the current state into qrhs (nodes 0..N); the state keeps
 * the filtered, averaged q, as the stage leaves it before its update. */
int astr_full_rhs(astr_full* fs, double* qrhs, const int64_t shape[3], const int64_t lbound[3], int where);
int astr_full_history(astr_full* fs, double* rows, int maxrows, int* nrows);

/* ---- checkpoint files: the reference's HDF5 flow field ---------------------------------- */
/* HDF5 files read and written by the library itself (the HDF5 library is not needed): the
 * reference's flow-field checkpoints and what the HDF5 library writes for its h5write calls
 * (superblock version 0, the root group as a symbol table, contiguous little-endian datasets).
 * Reading also takes superblocks version 1-3, version-2 object headers, compact link groups,
 * compact storage, float32 / integer / big-endian elements and a user block; chunked or
 * compressed datasets return ASTR_ERR_UNSUPPORTED. Host memory only; no context, no GPU.
 * Errors: ASTR_ERR_ARG (bad argument, missing dataset, shape mismatch), ASTR_ERR_STATE (I/O error,
 * malformed file), ASTR_ERR_UNSUPPORTED (a format feature outside the above). */
typedef struct astr_h5 astr_h5;
/* mode "write" creates or truncates the file; "read" opens it; "rdwr" opens an existing
 * version-0 file to add datasets (what h5srite does to the flow-field file). */
int astr_h5io_init(const char* filename, const char* mode, astr_h5** out);
/* Writes the group structures and the superblock (write, rdwr) and closes the file. */
int astr_h5io_end(astr_h5* h);
/* The message of the last failed call on h (h == NULL: of the last failed astr_h5io_init or
 * astr_h5io_end of this thread). */
const char* astr_h5_last_error(const astr_h5* h);
/* A dataset holding the Fortran array var of shape dims[0..rank-1] (first index fastest; the
 * HDF5 dataspace is the reversed shape, as the Fortran HDF5 interface stores it). */
int astr_h5write_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], const double* var);
int astr_h5write_i4(astr_h5* h, const char* varname, int rank, const int64_t dims[], const int32_t* var);
/* The block of Fortran shape dims at Fortran offsets offset[] (NULL: all zero) of a dataset of
 * rank `rank` (mode 'h', h5ra3d_r8_struct's hyperslab), or dims' element count from element
 * offset[0] of a one-dimensional dataset (mode 's', h5ra3d_r8_stream); a scalar dataset reads as
 * rank 1, dims {1}. Elements are converted to the output type; astr_h5read_i4 takes integer
 * datasets only. */
int astr_h5read_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], const int64_t offset[],
                   char mode, double* var);
int astr_h5read_i4(astr_h5* h, const char* varname, int rank, const int64_t dims[], const int64_t offset[],
                   char mode, int32_t* var);
/* Rank, Fortran-order shape (up to 32 entries), type class (0 integer, 1 float, -1 other) and
 * element size of a dataset. */
int astr_h5_dataset_info(astr_h5* h, const char* varname, int* rank, int64_t dims[], int* type_class,
                         int* type_size);
/* Members of the root group: their number and the i-th name (NUL-terminated, len bytes at most). */
int astr_h5_count(astr_h5* h, int* n);
int astr_h5_name(astr_h5* h, int i, char* name, int len);

/* The flow-field file of writeflfed: datasets ro, u1, u2, u3, p, t of Fortran shape (im+1, jm+1,
 * km+1) from the state's q by q2fvar (src/fludyna.F90:545-634, on the GPU), then nstep (integer)
 * and time (real(8)), one element each, the state's step counter and time. The conversions use
 * the state's stage buffers (no device allocation); the transfers go through 128 MB of pinned
 * host memory that the first checkpoint call of the process allocates and keeps, and up to 8
 * host threads for the duration of the call. A file of that name is replaced (the reference
 * moves the previous one aside first, bakupfile). */
int astr_state_write_flowfield(astr_state* st, const char* filename);
int astr_full_write_flowfield(astr_full* fs, const char* filename);
/* readcheckpoint's flow-field read and updateq: ro, u1, u2, u3, p, t (mode 'h': 3-D datasets of
 * Fortran shape (im+1, jm+1, km+1); 's': 1-D datasets of as many elements) and nstep, time; q =
 * fvar2q(ro, u, t) (src/fludyna.F90:449-533, the temperature branch, on the GPU); the state's step
 * counter and time are set from the file and returned in *nstep, *time when not NULL. */
int astr_state_read_flowfield(astr_state* st, const char* filename, char mode, int* nstep, double* time);
int astr_full_read_flowfield(astr_full* fs, const char* filename, char mode, int* nstep, double* time);

/* ---- no-allocation variant -------------------------------------------------------- */
/* dt such that cflcal's CFL equals `cfl` for the conserved variables q (a DEVICE array,
 * Fortran order q(lb.., 1:5) covering nodes 0..im x 0..jm x 0..km of a periodic box of side
 * 2*pi), like astr_cfl_dt but for callers that cannot let the library allocate device memory
 * (codes that run inside a fixed device pool or a capped allocator, where cudaMalloc fails or
 * synchronises the device mid-step). It has no counterpart in the reference.
 * It allocates nothing: its scratch is a 1.5 MB static device array that every GPU loading the
 * library holds until exit, which caps (jm+1)*(km+1) at 524288 (ASTR_ERR_UNSUPPORTED beyond).
 * The first call on a device looks the array's address up on that device. The call returns dt
 * to the host and so synchronises its stream: it cannot be made during stream capture (it
 * returns ASTR_ERR_ARG then). All calls share the array: calls that overlap on the GPU race.
 * ctx may be NULL (the caller's current device and its default stream, no message); otherwise
 * the call runs on ctx's device and stream, restores the caller's current device, and errors
 * set ctx's message. */
int astr_cfl_dt_noalloc(astr_ctx* ctx, const double* q, const int64_t shape[3], const int64_t lbound[3],
                        int im, int jm, int km, double mach, double gamma, double cfl, double* dt);

#ifdef __cplusplus
}
#endif
#endif
