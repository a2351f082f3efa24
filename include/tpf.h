/*
 * tpf.h -- C ABI of the B200 (sm_100a) implementation of TwoPhaseFlow's hot path:
 * the 6th-order combined compact difference (CCD) operator and the
 * variable-density FVM pressure-Poisson (PPE) solve.
 *
 * Plain C: opaque handles, device pointers, sizes, an explicit CUDA stream
 * (cudaStream_t passed as void*), int status codes.  No torch or C++ types.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   CCD: src/twophase/ccd/ccd_solver.py:79-281 (CCDSolver)
 *   PPE: src/twophase/ppe/interfaces.py:28-86 (IPPESolver.solve),
 *        src/twophase/ppe/fvm_matrixfree.py:46-363 (PPESolverFVMMatrixFree)
 *
 * Status codes mirror the reference's error conventions: the Python layer maps
 * TPF_EINVAL -> ValueError, TPF_ESINGULAR -> numpy.linalg.LinAlgError,
 * TPF_ENOCONV -> RuntimeError("did not converge ... info=<iters>"),
 * TPF_ECUDA / TPF_EABORT -> RuntimeError.
 *
 * Threading: calls on one handle are not thread safe; distinct handles are
 * independent.  All compute calls are asynchronous on `stream` unless stated.
 */
#ifndef TPF_H_
#define TPF_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum tpf_status {
  TPF_OK = 0,
  TPF_EINVAL = 1,     /* invalid argument (reference: ValueError)            */
  TPF_ENOCONV = 2,    /* Krylov did not converge (reference: RuntimeError)    */
  TPF_ECUDA = 3,      /* CUDA runtime error                                   */
  TPF_EABORT = 4,     /* a bounded device wait gave up (barrier timeout)      */
  TPF_ESINGULAR = 5   /* singular pivot in a factorization (LinAlgError)      */
};

enum tpf_dtype { TPF_F64 = 0, TPF_F32 = 1 };
enum tpf_bc { TPF_BC_WALL = 0, TPF_BC_PERIODIC = 1 };

/* flags for tpf_ccd_apply */
enum tpf_ccd_flags {
  TPF_CCD_APPLY_METRIC = 1   /* map xi-space derivatives to x (non-uniform grid) */
};

/* Library version (major*10000 + minor*100 + patch). */
int tpf_version(void);
/* Message of the last failing call on this host thread ("" if none). */
const char* tpf_last_error(void);

/* Launch-shape autotuning of the stencil kernels whose results do not
 * depend on the launch shape (no counterpart in the reference): the CLS flux
 * divergence and Rhie-Chow march kernels (nodes per thread along the axis)
 * and the reinitialization's Crank-Nicolson line solves on the strided axes
 * (threads per block).  The first call of a signature (kernel, shape, dtype)
 * outside stream capture times every candidate on scratch memory and keeps
 * the fastest for the process; results are bit-for-bit those of any other
 * shape.  mode 1 (default) tunes; 0 switches tuning off and forgets the
 * choices (the heuristic shapes are then used); 2 + k makes every tuned
 * kernel take its candidate k (clamped to its last one) without timing, to
 * check that every shape gives the same bits.  The CCD plans carry their own
 * autotuner (tpf_ccd_plan_set_autotune). */
int tpf_set_launch_autotune(int mode);
/* Number of signatures tuned so far in this process. */
int tpf_launch_autotune_entries(void);

/* ------------------------------------------------------------------------ */
/* CCD operator                                                              */
/* ------------------------------------------------------------------------ */
typedef struct tpf_ccd_plan tpf_ccd_plan;

/* One axis of a CCD operator: n_pts nodes (N+1), spacing h (the stencil
 * spacing: L/N on uniform grids, 1/N in xi-space), boundary TPF_BC_WALL or
 * TPF_BC_PERIODIC, data type TPF_F64 or TPF_F32.
 * Replaces CCDSolver._get_axis_solver / build_ccd_axis_solver /
 * build_ccd_axis_solver_periodic (ccd_solver.py:99-130,294-299;
 * ccd_solver_helpers.py:227-314,406-423).  Wall requires n_pts >= 6
 * (ccd_solver.py:459-465) -> TPF_EINVAL; periodic requires n_pts >= 4.
 * Blocking (host-side factorization + one host->device copy). */
int tpf_ccd_plan_create(tpf_ccd_plan** plan, int64_t n_pts, double h, int bc,
                        int dtype);
int tpf_ccd_plan_destroy(tpf_ccd_plan* plan);

/* Launch-shape autotuning of the line kernels (default on; no counterpart
 * in the reference): the first tpf_ccd_apply of each (line count, axis kind,
 * boundary, outputs, dtype) combination times a few launch shapes on the
 * caller's stream and keeps the fastest -- warps per block and tile ring depth
 * of the lane-per-line kernel (3-D grids), lines per block and tile buffers of
 * the warp kernel (2-D grids) -- results are identical for every shape.  That first call synchronizes the stream; it is skipped while the
 * stream is being captured.  enable = 0 switches tuning off and forgets the
 * choices. */
int tpf_ccd_plan_set_autotune(tpf_ccd_plan* plan, int enable);

/* Metric of a non-uniform axis (host arrays of n_pts doubles: J = dxi/dx and
 * dJ/dxi).  Replaces the grid metric used by apply_ccd_metric
 * (ccd_solver_helpers.py:509-533).  Blocking. */
int tpf_ccd_plan_set_metric(tpf_ccd_plan* plan, const double* J,
                            const double* dJ);

/* d1/d2 of f along the plan's axis for an array viewed as C-order
 * [outer, n_pts, inner] (the axis in the middle).  f, d1, d2 are device
 * pointers of the plan's dtype (f must not alias d1 or d2 -> TPF_EINVAL);
 * d1 or d2 may be NULL (first_derivative /
 * second_derivative).  bc_left / bc_right: optional host pointers to
 * (f'_b, f''_b) overrides of the wall closure (testing hook of the reference),
 * NULL for the compact closure.  flags: TPF_CCD_APPLY_METRIC.
 * Replaces CCDSolver.differentiate / first_derivative / second_derivative /
 * differentiate_raw (ccd_solver.py:134-237; ccd_solver_helpers.py:38-224,
 * 426-506). */
int tpf_ccd_apply(const tpf_ccd_plan* plan, int64_t outer, int64_t inner,
                  const void* f, void* d1, void* d2, const double* bc_left,
                  const double* bc_right, int flags, void* stream);

/* FP32 line solves under FP64 iterative refinement (no counterpart in the
 * reference, whose CCD is FP64): d1, d2 (FP64) of the FP64 field f along the
 * plans' axis, viewed as [outer, n_pts, inner].  The FP32 plan solves the
 * FP32-rounded field; then `refinements` times (0..8) the residual of the
 * full CCD system (interior Eq-I/Eq-II rows and the one-sided wall closures,
 * ccd_solver.py:11-22,408-465) is formed in FP64 and an FP32 correction solve
 * of the folded system is added in FP64.  Both plans: the same n_pts and h,
 * TPF_BC_WALL, dtypes TPF_F64 and TPF_F32.  work: device scratch of
 * 5 * outer * n_pts * inner floats.  The first call builds the plan's FP32
 * per-row factors (a host factorization and one allocation). */
int tpf_ccd_apply_refined(const tpf_ccd_plan* p64, const tpf_ccd_plan* p32, int64_t outer, int64_t inner,
                          const double* f, double* d1, double* d2, int refinements, float* work, void* stream);

/* Variable-density CCD term along the plan's axis, fused into the line
 * solve's output stage: out (+)= D2 f / rho - (drho / rho^2) D1 f, where drho
 * is d(rho)/dx along this axis (accumulate != 0 adds to out).  Summed over
 * the axes this is the CCD operator L_H p = sum_a [D2_a p / rho -
 * (D1_a rho / rho^2) D1_a p].  Replaces compute_ccd_laplacian
 * (ppe/ccd_ppe_utils.py:51-82). */
int tpf_ccd_apply_vd(const tpf_ccd_plan* plan, int64_t outer, int64_t inner,
                     const void* f, const void* rho, const void* drho,
                     void* out, int accumulate, int flags, void* stream);

/* Velocity corrector fused into the CCD line solve
 * (VelocityCorrector.correct with ccd_pressure_gradient,
 * src/twophase/coupling/velocity_corrector.py:41-89):
 *   u_out = u_star - (dt / rho) * dp/dx_axis
 * with dp/dx_axis the CCD first derivative of pres along the plan's axis
 * (metric applied when TPF_CCD_APPLY_METRIC), taken as 0 on wall planes
 * (enforce_wall_neumann), i.e. u_out = u_star there.  u_out may be u_star
 * (in place); pres must not alias the other arrays.  Dtype of the plan. */
int tpf_ccd_apply_corrector(const tpf_ccd_plan* plan, int64_t outer, int64_t inner,
                            const void* pres, const void* u_star, const void* rho, double dt,
                            void* u_out, int flags, void* stream);

/* CFL maxima (CFLCalculator.compute, src/twophase/time_integration/cfl.py:85-137):
 * out[c] = max |comps[c][i]| for the ncomp (1..3) velocity components and, when
 * mu and rho are given, out[3] = max mu[i] / rho[i] (values assumed >= 0; a
 * NaN propagates).  n values each, dtype TPF_F64 / TPF_F32; out is a device
 * array of 4 doubles (zeroed by the call); asynchronous on stream.  The time
 * step itself is the host formula of the reference on these maxima. */
int tpf_cfl_maxima(int64_t n, int ncomp, const void* const* comps, const void* mu, const void* rho,
                   int dtype, double* out, void* stream);

/* DCCD dissipative filter (src/twophase/levelset/curvature.py:60-127): for
 * each axis in turn f <- f + c (f[+1] - 2 f + f[-1]) on nodes 1..N-1 (wall)
 * or on the N unique nodes with wrap-around, image node N <- node 0
 * (periodic[axis] != 0); c = eps, or eps * sw[node] when sw is given; then
 * the wall planes take the unfiltered input.  shape: nodes per axis (ndim 2
 * or 3, C order); f and out distinct.  tmp: workspace of f's size, distinct
 * from f, out and sw, needed in 3-D (2-D runs both passes in one kernel and
 * ignores it; NULL allowed there). */
int tpf_dccd_filter(int ndim, const int64_t* shape, const int* periodic, double eps, const void* sw,
                    const void* f, void* out, void* tmp, int dtype, void* stream);

/* Curvature from psi (CurvatureCalculatorPsi.compute, curvature_psi.py:72-173)
 * given its CCD derivatives: d1[a], d2[a] per axis and the mixed derivatives
 * (2-D: mixed[0] = psi_xy; 3-D: xy, xz, yz); kappa = 0 where
 * psi <= psi_min or psi >= 1 - psi_min.  n values each. */
int tpf_curvature_psi(int ndim, int64_t n, const void* psi, const void* const* d1, const void* const* d2,
                      const void* const* mixed, double psi_min, void* kappa, int dtype, void* stream);

/* 3x3 Gaussian [1 2 1; 2 4 2; 1 2 1] / 16 with edge replication, 2-D n0 x n1
 * (curvature_psi.py:176-197); in and out distinct. */
int tpf_gaussian3x3(int64_t n0, int64_t n1, const void* in, void* out, int dtype, void* stream);

/* rho = rho_g + (rho_l - rho_g) psi and mu = mu_g + (mu_l - mu_g) psi
 * (update_properties, src/twophase/levelset/heaviside.py:167-187); either
 * output may be NULL. */
int tpf_update_properties(int64_t n, const void* psi, double rho_l, double rho_g, double mu_l, double mu_g,
                          void* rho, void* mu, int dtype, void* stream);

/* One axis of the Rhie-Chow face-velocity divergence
 * (RhieChowInterpolator.face_velocity_divergence / _rc_flux_1d /
 * _flux_divergence_1d, src/twophase/spatial/rhie_chow.py:55-284).  shape:
 * nodes per axis (C order); h = L/N of the axis; dp = the CCD first
 * derivative of p along the axis (its boundary values are replaced by
 * one-sided differences on a wall axis, periodic = 0).  kappa, psi and dpsi
 * (= CCD D1 psi along the axis) all NULL, or all given with we != 0 for the
 * balanced-force form.  div = this axis' divergence (accumulate = 0, the first
 * axis) or div + it (accumulate = 1). */
int tpf_rc_divergence_axis(int ndim, const int64_t* shape, int axis, int periodic, double h, double dt,
                           const void* u_star, const void* p, const void* rho, const void* dp,
                           const void* kappa, const void* psi, const void* dpsi, double we,
                           int accumulate, void* div, int dtype, void* stream);

/* ---- CLS transport: FCCD flux-form advection and TVD-RK3 --------------- */

/* prod = u * phi, n values (the product of compute_fccd_flux_contribution,
 * src/twophase/ccd/fccd_advection_helpers.py:8-13). */
int tpf_fccd_product(int64_t n, const void* u, const void* phi, void* prod, int dtype, void* stream);

/* acc (+)= -face_divergence(face_value(prod, q)) along one axis
 * (fccd_advection_helpers.py:8-13; fccd.py:213-233,279-299,464-520): face
 * value 0.5 (p_j + p_{j+1}) - (H^2/16)(q_j + q_{j+1}), divergence
 * (F_k - F_{k-1}) / H on the N unique nodes with wrap-around and node N <-
 * node 0 (periodic) or on nodes 1..N-1 with 0 on the wall nodes.  q = the CCD
 * second derivative of prod along the axis; h = the uniform node spacing.
 * accumulate = 0 writes 0 + (-div) (the first axis), 1 adds to acc.  acc must
 * not alias prod or q. */
/* Option C node gradient along one axis (FCCDSolver.node_gradient,
 * fccd.py:392-462, with the face gradient of :243-277): face gradients
 * (u_{j+1} - u_j)/H - (H/24)(q_{j+1} - q_j), then at the nodes
 * 0.5 (d_L + d_R) - (H/16)(q_{i+1} - q_{i-1}); wall nodes 0 and N take their
 * one face gradient; periodic axes wrap over the N unique nodes and node N
 * repeats node 0.  q = the CCD second derivative of u along the axis.
 * mode 0: out = gradient; 1: out = 0 - uk * gradient; 2: out -= uk *
 * gradient (the nodal advection sum, fccd_advection_helpers.py:46-72).
 * out must not alias u, q or uk. */
int tpf_fccd_node_gradient_axis(int ndim, const int64_t* shape, int axis, int periodic, double h, const void* u,
                                const void* q, const void* uk, int mode, void* out, int dtype, void* stream);
/* The same on a non-uniform axis (the reference's array weights,
 * fccd_helpers.py:8-52): face_inv_h[f] = 1/H_f and face_h_24[f] = H_f/24 for
 * the N faces (H_f = x_{f+1} - x_f), node_h_16[i] = H_node_i/16 for the N+1
 * nodes (H_node = (H_{i-1} + H_i)/2 inside, H_0 and H_{N-1} at the ends);
 * device arrays in FP64. */
int tpf_fccd_node_gradient_axis_nonuniform(int ndim, const int64_t* shape, int axis, int periodic,
                                           const double* face_inv_h, const double* face_h_24,
                                           const double* node_h_16, const void* u, const void* q, const void* uk,
                                           int mode, void* out, int dtype, void* stream);
int tpf_fccd_flux_divergence_axis(int ndim, const int64_t* shape, int axis, int periodic, double h,
                                  const void* prod, const void* q, int accumulate, void* acc, int dtype,
                                  void* stream);
/* The same on a non-uniform axis (fccd.py:279-299,464-520 with array
 * weights): face_h2_16[f] = H_f H_f / 16 for the N faces; node_inv_width =
 * 1 / ((H_{i-1} + H_i)/2) for the interior nodes i = 1..N-1 of a wall axis
 * (N-1 values) or for the N unique nodes of a periodic axis (H_{-1} = H_{N-1});
 * device arrays in FP64. */
int tpf_fccd_flux_divergence_axis_nonuniform(int ndim, const int64_t* shape, int axis, int periodic,
                                             const double* face_h2_16, const double* node_inv_width,
                                             const void* prod, const void* q, int accumulate, void* acc, int dtype,
                                             void* stream);

/* One TVD-RK3 stage (src/twophase/time_integration/tvd_rk3.py:26-48) with the
 * post-stage clip to [lo, hi] (clip != 0) and periodic image sync of
 * FCCDLevelSetAdvection.advance (levelset/fccd_advection.py:86-129):
 * stage 1: out = q + dt L; stages 2 and 3: out = ca q0 + cb (q + dt L)
 * (ca, cb = 0.75, 0.25 and 1/3, 2/3).  periodic[a] != 0 marks periodic axes
 * (their node N takes node 0's value); with any periodic axis out must not
 * alias an input. */
int tpf_tvd_rk3_stage(int ndim, const int64_t* shape, const int* periodic, int stage, double ca, double cb,
                      double dt, const void* q0, const void* q, const void* L, int clip, double lo, double hi,
                      void* out, int dtype, void* stream);

/* In place: node N of every periodic axis takes node 0's value, axes in turn
 * (sync_periodic_image_nodes, src/twophase/core/boundary.py:116-133). */
int tpf_sync_periodic_images(int ndim, const int64_t* shape, const int* periodic, void* arr, int dtype,
                             void* stream);

/* UCCD6 convection, one (component j, axis k) term
 * (UCCD6ConvectionTerm.compute, src/twophase/ns_terms/uccd6_convection.py:83-128):
 * acc = (first ? 0 : acc) - 0.5 (uk d1 + cons), then acc - coeff (uref[0] d8);
 * d1 = CCD D1_k u_j, cons = CCD D1_k (u_k u_j), d8 = (CCD D2_k)^4 u_j,
 * uref = max |u_k| on the device (tpf_cfl_maxima), coeff = sigma h_k^7. */
int tpf_uccd6_accumulate(int64_t n, int first, const void* uk, const void* d1, const void* cons, const void* d8,
                         double coeff, const double* uref, void* acc, int dtype, void* stream);

/* ---- Split reinitialization (src/twophase/levelset/reinit_split.py:73-102) */

/* flux[a] = psi (1 - psi) d1[a] / max(sqrt(max(|d1|^2, 1e-12)), 1e-6), a < ndim
 * (compute_gradient_normal + dccd_compression_div, levelset/reinit_ops.py:57-114);
 * d1[a] = the CCD first derivative of psi along axis a.  n values each. */
int tpf_reinit_compression_flux(int ndim, int64_t n, const void* psi, const void* const* d1, void* const* flux,
                                int dtype, void* stream);

/* div (+)= g + eps_d ((g[+1] - 2 g) + g[-1]) along one axis with one ghost
 * node each side: pad 0 = zero, 1 = periodic (g[n-2] / g[1]), 2 = the end
 * node (neumann, outflow) (filtered_divergence, reinit_ops.py:83-105;
 * pad_ghost_cells, core/boundary.py:249-292).  g = the CCD first derivative of
 * the axis' compression flux; accumulate = 0 writes 0 + it. */
int tpf_reinit_filtered_divergence_axis(int ndim, const int64_t* shape, int axis, int pad, double eps_d,
                                        const void* g, int accumulate, void* div, int dtype, void* stream);
/* The same on a non-uniform grid (filtered_divergence, reinit_ops.py:95-105):
 * g is the CCD derivative in xi-space (no metric) and each filtered value is
 * multiplied by J[k] (the metric of node k along the axis, FP64 device array)
 * before it is written or added. */
int tpf_reinit_filtered_divergence_axis_metric(int ndim, const int64_t* shape, int axis, int pad, double eps_d,
                                               const double* J, const void* g, int accumulate, void* div, int dtype,
                                               void* stream);

/* One CN-ADI half-step along one axis (cn_diffusion_axis, reinit_ops.py:169-204):
 * rhs = (M2 + mu B2) in with coefficients cR (off-diagonal), dR (diagonal)
 * and doubled off-diagonals on the end rows, then the Thomas sweep with the
 * factors f (n-1), m (n), sup (n-1) of build_cn_factors (:117-166), device
 * FP64 arrays.  in and out distinct. */
int tpf_reinit_cn_axis(int ndim, const int64_t* shape, int axis, double cR, double dR, const double* f,
                       const double* m, const double* sup, const void* in, void* out, int dtype, void* stream);

/* sums[0] = sum q dV, sums[1] = sum 4 q (1 - q) dV (two fixed-order passes;
 * partials: 2048 doubles of device workspace).  dV: FP64 control volumes. */
int tpf_mass_sums(int64_t n, const void* q, const double* dV, double* partials, double* sums, int dtype,
                  void* stream);

/* out = clip(q + gate * (target[0] - sums[0]) / W_safe * 4 q (1 - q), 0, 1),
 * W = sums[1], W_safe = W if W > 1e-12 else 1, gate = W > 1e-12
 * (apply_mass_correction, levelset/heaviside.py:118-149); all on the device. */
int tpf_mass_correction_apply(int64_t n, const void* q, const double* target, const double* sums, void* out,
                              int dtype, void* stream);

/* ---- Viscous stress divergence (src/twophase/ns_terms/viscous_spatial.py:28-153) */

/* total (+)= D_lo(v) along one axis, v = mu (a + b) (mu and b given) or a
 * (mu, b NULL), D_lo = _low_order_derivative (viscous_spatial.py:70-104):
 * (v_1 - v_0)/dx0 and (v_{n-1} - v_{n-2})/dxl at the ends,
 * cl[k-1] v_{k-1} + cc[k-1] v_k + cr[k-1] v_{k+1} inside (coefficients per
 * interior node, FP64 device arrays of n-2, as the reference forms them from
 * the node coordinates).  finalize = 1 then divides by Re rho (the last axis).
 * accumulate = 0 writes 0 + it.  total must not alias an operand. */
int tpf_visc_lowfd_axis(int ndim, const int64_t* shape, int axis, const double* cl, const double* cc,
                        const double* cr, double dx0, double dxl, const void* a, const void* b, const void* mu,
                        int accumulate, int finalize, const void* rho, double re, void* total, int dtype,
                        void* stream);

/* out = mu (a + b), n values (the stress of the legacy CCD scheme). */
int tpf_visc_stress(int64_t n, const void* mu, const void* a, const void* b, void* out, int dtype, void* stream);

/* Interface-band form of the ccd_bulk viscous scheme, used when psi is given
 * (ViscousSpatialEvaluator.evaluate, ns_terms/viscous_spatial.py:50-64,
 * 158-221).  tpf_visc_band_masks: band[i] = 1 where any node of the 3^ndim box
 * around i (inside the domain) has 1e-6 < psi < 1 - 1e-6
 * (_interface_band_mask); normal[a][i] = 1 where |grads[a]| is the largest
 * of the axes' |grads| and that maximum exceeds 1e-14, or where the maximum
 * is <= 1e-14 (_normal_axis_masks); grads = the low-order derivatives of psi
 * (tpf_visc_lowfd_axis).  Masks are one byte per node.
 * tpf_visc_select: s = mask ? lo : hi (lo when mask is NULL, hi may then be
 * NULL); mode 0 out = s, 1 out += s, 2 out = 0 + s.
 * tpf_visc_band_finalize: out = (band ? nt : mu lap) / (Re rho). */
int tpf_visc_band_masks(int ndim, const int64_t* shape, const void* psi, const void* const* grads,
                        unsigned char* band, unsigned char* const* normal, int dtype, void* stream);
int tpf_visc_select(int64_t n, const unsigned char* mask, const void* lo, const void* hi, int mode, void* out,
                    int dtype, void* stream);
int tpf_visc_band_finalize(int64_t n, const unsigned char* band, const void* nt, const void* lap, const void* mu,
                           const void* rho, double re, void* out, int dtype, void* stream);

/* total (+)= g, then (finalize) total / (Re rho). */
int tpf_visc_accumulate(int64_t n, const void* g, int accumulate, int finalize, const void* rho, double re,
                        void* total, int dtype, void* stream);

/* Predictor combinations (PicardCNAdvance.advance,
 * src/twophase/time_integration/cn_advance/picard_cn.py:43-96; the explicit
 * branch of ViscousTerm.apply_cn_predictor, ns_terms/viscous.py:161-167):
 * mode 0: out = u + dt (e / rho + vn); mode 1: out = u + dt ((e / rho + 0.5 vn)
 * + 0.5 vs); mode 2 (the explicit branch of Predictor.compute,
 * time_integration/ab2_predictor.py:196-201): out = u + dt (e + rho vn) / rho;
 * mode 3 (RichardsonCNAdvance.advance, cn_advance/richardson_cn.py:76-109):
 * out = (4 u - vn) / 3 with u the two half steps and vn the full step (e, rho,
 * vs unused, may be NULL).  e = explicit right-hand side, vn / vs = viscous
 * force at u and at the predicted state.  n values each; out may alias u. */
int tpf_cn_predictor_combine(int64_t n, int mode, double dt, const void* u, const void* e, const void* rho,
                             const void* vn, const void* vs, void* out, int dtype, void* stream);

/* ---- AB2 + IPC momentum predictor (time_integration/ab2_predictor.py:110-209) */

/* acc = (first ? 0 : acc) - u du (ConvectionTerm.compute, ns_terms/convection.py:43-82). */
int tpf_ns_conv_accumulate(int64_t n, int first, const void* u, const void* du, void* acc, int dtype, void* stream);

/* mode 0: out = -a / s (GravityTerm, s = Fr^2, ns_terms/gravity.py:53-86);
 * mode 1: out = (a b) / s (SurfaceTensionTerm CSF kappa dpsi / We,
 * ns_terms/surface_tension.py:48-96); mode 2: out = a / s (b unused). */
int tpf_ns_scaled(int64_t n, int mode, const void* a, const void* b, double s, void* out, int dtype, void* stream);

/* out = ((rho c + grav) + st) + (-gradp), c = 1.5 conv_n - 0.5 conv_prev (ab2)
 * or conv_n; grav / st NULL add +0 (the reference's zero arrays). */
int tpf_ns_explicit_rhs(int64_t n, int ab2, const void* conv_n, const void* conv_prev, const void* rho,
                        const void* grav, const void* st_force, const void* gradp, void* out, int dtype,
                        void* stream);

/* Zero grad at index 0 and n_pts-1 along the axis of a [outer, n, inner]
 * array (wall axes only; no-op for periodic plans).  Replaces
 * CCDSolver.enforce_wall_neumann (ccd_solver.py:264-281;
 * ccd_boundary_helpers.py:52-61). */
int tpf_ccd_enforce_wall_neumann(const tpf_ccd_plan* plan, int64_t outer,
                                 int64_t inner, void* grad, void* stream);

/* ------------------------------------------------------------------------ */
/* Variable-density FVM PPE                                                   */
/* ------------------------------------------------------------------------ */
typedef struct tpf_ppe tpf_ppe;

enum tpf_ppe_method {
  TPF_PPE_CG = 0,        /* CG on the control-volume-weighted SPD system       */
  TPF_PPE_GMRES = 1      /* restarted GMRES, left preconditioned               */
};
enum tpf_ppe_precond {
  TPF_PRECOND_NONE = 0,
  TPF_PRECOND_JACOBI = 1,
  TPF_PRECOND_LINE = 2,       /* shifted additive line solves, exact Thomas   */
  TPF_PRECOND_LINE_PCR = 3    /* same, PCR truncated to pcr_stages stages: the
                               * reference's GPU line solver
                               * (linalg_backend.py:77-163)                      */
};
enum tpf_precision {
  TPF_PREC_F64 = 0,      /* FP64 Krylov                                          */
  TPF_PREC_MIXED = 1     /* FP32 inner CG under FP64 iterative refinement       */
};

typedef struct tpf_ppe_options {
  int method;            /* tpf_ppe_method                                      */
  int precond;           /* tpf_ppe_precond                                     */
  int precision;         /* tpf_precision                                       */
  double tol;            /* relative residual tolerance (pseudo_tol)             */
  int64_t maxiter;       /* CG: iterations; GMRES: restart cycles (pseudo_maxiter)*/
  int restart;           /* GMRES restart length (ppe_restart)                   */
  double c_tau;          /* line-preconditioner shift factor (pseudo_c_tau)      */
  int pcr_stages;        /* TPF_PRECOND_LINE_PCR stages (ppe_pcr_stages)         */
  double inner_tol;      /* MIXED: FP64 residual replacement + FP32 CG restart     
                          * whenever ||r|| fell by this factor (default 1e-3)   */
  int64_t max_refine;    /* reserved                                             */
} tpf_ppe_options;

typedef struct tpf_ppe_result {
  int64_t iterations;    /* CG iterations / GMRES inner iterations (all sweeps)  */
  int64_t applies;       /* operator applications                                */
  int64_t refinements;   /* MIXED: FP64 residual replacements                    */
  double rel_residual;   /* ||b - A x|| / ||b|| of the solved system             */
  int info;              /* 0 converged, >0 iteration budget exhausted           */
} tpf_ppe_result;

/* Fill `opts` with the reference defaults: GMRES, line preconditioner,
 * tol 1e-8, maxiter 500, restart 80, c_tau 2, pcr_stages 4
 * (fvm_matrixfree.py:90-127; config.py:331-333). */
void tpf_ppe_default_options(tpf_ppe_options* opts);

/* Handle for one wall-bounded grid: ndim in {2,3}, N[a] cells per axis,
 * coords[a] = host array of N[a]+1 node coordinates, pin = flat index of the
 * gauge-pinned node (BoundarySpec.pin_dof).  Allocates the device workspace.
 * Replaces PPESolverFVMMatrixFree.__init__ / _refresh_grid_metrics
 * (fvm_matrixfree.py:66-138,338-343; fvm_matrixfree_helpers.py:23-43). */
int tpf_ppe_create(tpf_ppe** h, int ndim, const int64_t* N,
                   const double* const* coords, int64_t pin,
                   const tpf_ppe_options* opts);
int tpf_ppe_destroy(tpf_ppe* h);
int tpf_ppe_set_options(tpf_ppe* h, const tpf_ppe_options* opts);
/* Kernel of the CG solve (same iteration, same stopping rule):
 * 0 (default) = the band-resident kernel when it applies, else 3 for FP64
 *     systems, else (mixed precision) 1;
 * 1 = one persistent cooperative launch with every vector in global memory
 *     (any grid, FP64 or mixed);
 * 2 = the band-resident kernel: 2-D systems whose nodes, split into one
 *     contiguous range per SM (at least one row each, at most 768 nodes per
 *     row), fit in shared memory with 12 FP64 vectors (~550^2 on a B200) or,
 *     mixed, 11 FP32 vectors and x in FP64 (~770^2); only the ranges' first
 *     and last rows cross L2 each iteration.
 *     TPF_EINVAL from tpf_ppe_solve when it does not apply;
 * 3 = streaming (FP64): each iteration as two ordinary full-occupancy
 *     kernels (vector update; stencil + inner products, the last block
 *     advancing the scalars on the device), chunks of 32 iterations
 *     replayed from a CUDA graph.  The mixed-precision route keeps 1. */
int tpf_ppe_set_cg_kernel(tpf_ppe* h, int kind);

/* Stream capture (no counterpart in the reference, which has no CUDA graphs):
 * tpf_ppe_solve with method TPF_PPE_CG may be called while `stream` is being
 * captured into a CUDA graph.  The whole solve is then recorded in the graph
 * (the persistent kernels as one cooperative launch; the streaming PCG as a
 * conditional WHILE node whose body runs 32 iterations and re-tests the
 * device-side convergence state), nothing is read back, and the result
 * fields are -1.  After a replay, tpf_ppe_read_result synchronizes `stream`
 * and returns that replay's result and status (TPF_ENOCONV as tpf_ppe_solve).
 * The GMRES route reads its residual on the host and returns TPF_EINVAL under
 * capture. */
int tpf_ppe_read_result(tpf_ppe* h, void* stream, tpf_ppe_result* result);

/* Build face coefficients, Jacobi diagonal and line-preconditioner state
 * from rho (device, grid shape, FP64).  Replaces prepare_operator /
 * _prepare_preconditioner_state (fvm_matrixfree.py:262-279,352-363;
 * fvm_matrixfree_helpers.py:46-104). */
int tpf_ppe_prepare(tpf_ppe* h, const double* rho, void* stream);

/* out = L p with the pinned row (out[pin] = p[pin]).  Replaces
 * PPESolverFVMMatrixFree.apply (fvm_matrixfree.py:281-300). */
int tpf_ppe_apply(tpf_ppe* h, const double* p, double* out, void* stream);

/* z = M^-1 r for the handle's preconditioner on the unweighted system.
 * Replaces apply_line_preconditioner / apply_jacobi_preconditioner
 * (fvm_matrixfree.py:302-331). */
int tpf_ppe_precondition(tpf_ppe* h, const double* r, double* z, void* stream);

/* Solve L p = rhs for the density given to the last tpf_ppe_prepare (or
 * prepare from `rho` first when rho != NULL).  p_init may be NULL.  p is
 * written with p[pin] = 0.  Synchronizes `stream` (the result is read back).
 * Returns TPF_ENOCONV when the iteration budget ends before tol (p holds the
 * last iterate).  Replaces PPESolverFVMMatrixFree.solve
 * (fvm_matrixfree.py:150-260) and the SciPy Krylov loops it calls
 * (gmres_helpers.py:16-80). */
int tpf_ppe_solve(tpf_ppe* h, const double* rhs, const double* rho, double* p,
                  const double* p_init, void* stream, tpf_ppe_result* result);

/* Batched solve (no counterpart in the reference, which solves one system
 * per call): n independent systems (n <= 64, each its own handle and grid,
 * all with method TPF_PPE_CG and one precision).  When every system is 2-D
 * and all their bands fit in shared memory at once (the systems' nodes
 * summing to at most ~340 000 in FP64, ~640 000 mixed, on 148 SMs): ONE
 * cooperative launch in which every system runs the band-resident PCG on its
 * own share of the SMs (proportional to ndof^1.5, its expected work) with its
 * own grid barrier.  Otherwise, FP64: the batched streaming PCG -- every
 * system's iterations in the same two launches (each system its own blocks,
 * threads in proportion to its nodes, its own scalars; a system's blocks
 * return once it is done), chunks of 32 iterations replayed from a CUDA
 * graph; mixed precision: one cooperative launch of the all-global body.
 * tpf_ppe_set_cg_kernel on any handle selects: 1 the all-global body, 2 the
 * band-resident batch (TPF_EINVAL if it does not fit), 3 the batched
 * streaming PCG (FP64 only; TPF_EINVAL for mixed precision or with another
 * handle asking for 1 or 2).  rho may be NULL (or hold NULL entries) for
 * handles prepared beforehand.  results[c] as tpf_ppe_solve; returns the
 * first failure (TPF_ENOCONV / TPF_EABORT) after all systems finished.
 * Synchronizes `stream`. */
int tpf_ppe_solve_batched(tpf_ppe* const* handles, int n, const double* const* rhs, const double* const* rho,
                          double* const* p, void* stream, tpf_ppe_result* results);

/* ---- FCCD matrix-free PPE ----------------------------------------------
 *
 * Replaces PPESolverFCCDMatrixFree on its default path
 * (src/twophase/ppe/fccd_matrixfree.py:105-611: constructor :117-215, apply
 * :378-398, operator core :400-428, solve :506-611, wall divergence
 * :762-829; face gradient src/twophase/ccd/fccd.py:243-277; Jacobi inverse
 * ppe/fccd_matrixfree_helpers.py:251-265): phase-density face coefficients
 * 2/(rho_L + rho_R), no interface coupling, full boundary faces, the legacy
 * operator pairing, SciPy GMRES (ppe/gmres_helpers.py:16-80) with the Jacobi
 * or no preconditioner.  Uniform grids; every axis wall or periodic. */
typedef struct tpf_fccd_ppe tpf_fccd_ppe;

typedef struct tpf_fccd_ppe_options {
  double tol;        /* GMRES relative tolerance (pseudo_tol, default 1e-8)        */
  int64_t maxiter;   /* GMRES restart cycles (pseudo_maxiter, default 500)          */
  int restart;       /* ppe_restart; 20 (SciPy's default) when the config has none  */
  int precond;       /* TPF_PRECOND_NONE (default) or TPF_PRECOND_JACOBI           */
} tpf_fccd_ppe_options;

void tpf_fccd_ppe_default_options(tpf_fccd_ppe_options* o);

/* ndim (2 or 3) axes of N[a] cells; coords[a]: HOST arrays of N[a]+1 node
 * coordinates (face weights H = x1 - x0, control-volume widths); h_ccd[a]:
 * the CCD spacing (L/N); periodic[a]: nonzero for a periodic axis; pin: the
 * pinned node (the reference's BoundarySpec.pin_dof, the centre node).
 * Allocates the handle's device state and one CCD plan per axis. */
int tpf_fccd_ppe_create(tpf_fccd_ppe** h, int ndim, const int64_t* N, const double* const* coords,
                        const double* h_ccd, const int* periodic, int64_t pin, const tpf_fccd_ppe_options* o);
int tpf_fccd_ppe_destroy(tpf_fccd_ppe* h);
int tpf_fccd_ppe_set_options(tpf_fccd_ppe* h, const tpf_fccd_ppe_options* o);
/* prepare_operator (fccd_matrixfree_lifecycle.py:44-95): keeps a device copy
 * of rho and forms the Jacobi inverse diagonal.  The first call also runs
 * one operator application (synchronizes `stream`). */
int tpf_fccd_ppe_prepare(tpf_fccd_ppe* h, const double* rho, void* stream);
/* out = L p with the pinned and periodic-image rows (apply, :378-398);
 * p and out distinct device arrays of the grid's nodes. */
int tpf_fccd_ppe_apply(tpf_fccd_ppe* h, const double* p, double* out, void* stream);
/* the Jacobi inverse diagonal of the last prepare, into out */
int tpf_fccd_ppe_diag_inv(tpf_fccd_ppe* h, double* out, void* stream);
/* solve (:506-611): prepare(rho), GMRES on the rhs with the pinned and image
 * rows zeroed, p[pin] = 0, images synchronised.  Synchronizes `stream`;
 * TPF_ENOCONV when GMRES does not converge (info = maxiter). */
int tpf_fccd_ppe_solve(tpf_fccd_ppe* h, const double* rhs, const double* rho, double* p, const double* p_init,
                       void* stream, tpf_ppe_result* result);

/* ---- allocation-free CG solve (no counterpart in the reference) ----------
 *
 * For callers that cannot allocate device memory while they run: a host whose
 * caching allocator (PyTorch's, a memory pool) already holds the device
 * memory, so a cudaMalloc inside a time step may fail or stall, or a solver
 * loop whose memory budget is fixed at start-up.  Same solve as tpf_ppe_solve
 * with method TPF_PPE_CG, precision TPF_PREC_F64 and precond TPF_PRECOND_JACOBI
 * or TPF_PRECOND_NONE (identical iterates), but no handle: the workspace is a
 * fixed file-scope device array of about 9.3 MB inside the library, and the
 * call issues no cudaMalloc / cudaFree and calls no allocating library.
 *
 * Limits: at most TPF_PPE_STATIC_MAX_DOF nodes in total (e.g. 256 x 256 cells
 * in 2-D, 39 x 39 x 39 cells in 3-D) and TPF_PPE_STATIC_MAX_AXIS nodes per
 * axis; larger grids are rejected with TPF_EINVAL (use tpf_ppe_create /
 * tpf_ppe_solve).  coords[a] are HOST arrays of N[a]+1 node coordinates (as
 * for tpf_ppe_create); rhs, rho, p, p_init are device arrays of the grid's
 * nodes.
 *
 * Set-up: the first call on a device (with that device current) looks up the
 * workspace's device address and keeps it for later calls on that device.
 * Under CUDA's lazy module loading that lookup is also what loads the module
 * holding the array, so the array's device memory is reserved by that first
 * call: make it at start-up, before any stream capture and before a fixed
 * memory budget is measured.  The kept address is not valid after
 * cudaDeviceReset on that device; the entry point must not be used after one.
 *
 * All calls on one device share the workspace, which keeps the last call's
 * contents (each call initialises what it reads): calls that overlap in time
 * on the same device (two host threads, or two streams without ordering
 * between them) race and must be serialised by the caller.  The call waits
 * for `stream` to drain before it returns (it reads the solve status back);
 * returns TPF_ENOCONV like tpf_ppe_solve. */
#define TPF_PPE_STATIC_MAX_DOF 66049
#define TPF_PPE_STATIC_MAX_AXIS 4097
int tpf_ppe_solve_cg_static(int ndim, const int64_t* N, const double* const* coords,
                            int64_t pin, const double* rhs, const double* rho, double* p,
                            const double* p_init, int precond, double tol,
                            int64_t maxiter, void* stream, tpf_ppe_result* result);

/* ------------------------------------------------------------------------ */
/* Learned PPE preconditioner (no counterpart in the reference, which has no  */
/* learned component; its PPE Krylov loops are SciPy cg / gmres,              */
/* src/twophase/ppe/gmres_helpers.py:16-80)                                   */
/* ------------------------------------------------------------------------ */
typedef struct tpf_unet tpf_unet;

/* Number of FP32 parameters of the U-Net (4 levels, 3x3 convolutions,
 * channels 16-32-64-128, 1x1 output).  Flat layout: for each of the 14
 * convolutions W[cout][cin][3][3] then b[cout]; then w_out[16], b_out. */
int64_t tpf_unet_num_params(void);

/* Network workspace for images of H x W nodes (multiples of 8) and batches
 * up to max_batch.  Parameters start at zero. */
int tpf_unet_create(tpf_unet** net, int H, int W, int max_batch);
int tpf_unet_destroy(tpf_unet* net);
/* Copy the FP32 master parameters in / out (host or device pointer). */
int tpf_unet_set_params(tpf_unet* net, const float* params, int on_device);
int tpf_unet_get_params(tpf_unet* net, float* params, int on_device);
/* How the forward pass is launched: 0 (default; -1 restores it) = one launch
 * per layer, programmatic dependent launch between them; 1 = the whole
 * network in one persistent cooperative launch (one CTA per SM, grid
 * barriers between layers, deep layers' output channels split over CTAs).
 * Both give the same outputs bit for bit; the persistent launch is faster
 * for a stand-alone call, the layered one inside a CUDA graph. */
int tpf_unet_set_forward_mode(tpf_unet* net, int mode);

/* y[B][H][W] = UNet(in2[B][H][W][4]) (device FP32; BF16 inside).  The four
 * input channels: scaled residual, density feature, and the scaled couplings
 * of the operator to the next row / column.  Synchronizes. */
int tpf_unet_forward(tpf_unet* net, int B, const float* in2, float* y, void* stream);
/* Parameter gradients (FP32, num_params, device) of sum(dy * y) for the
 * activations of the last tpf_unet_forward with the same B.  Synchronizes. */
int tpf_unet_backward(tpf_unet* net, int B, const float* dy, float* grads, void* stream);
/* One Adam step on the mean over the batch of the relative squared error
 * sum (y - target)^2 / sum target^2; *loss (may be NULL) is that mean before
 * the step.  Synchronizes when loss != NULL. */
int tpf_unet_train_step(tpf_unet* net, int B, const float* in2, const float* target, float lr,
                        float weight_decay, double* loss, void* stream);

/* One Adam step on the energy loss of a coarse-grid correction (two-level
 * training): per sample, with y the network output, x = in2[..,0] and
 * A~ = I - couplings (coupl[q][0] to the next row, coupl[q][1] to the next
 * column, inside the nc0 x nc1 coarse grid),
 * L = (y.A~y - 2 y.x) / escale + 1, the relative A-norm error left after the
 * correction; *loss (may be NULL) is the batch mean before the step. */
int tpf_unet_train_step_energy(tpf_unet* net, int B, const float* in2, const float* coupl, const double* escale,
                               int nc0, int nc1, float lr, float weight_decay, double* loss, void* stream);

/* Defaults (tpf_lppe_default_options): tol 1e-8, maxiter 2000, smooth 16,
 * omega 0.8, check_every 8, stall_checks 16, stall_factor 0.5, fallback 1,
 * use_graph 1, window 8, outer 1 (flexible GMRES), restart 60. */
typedef struct tpf_learned_options {
  double tol;           /* relative residual tolerance of the weighted system   */
  int64_t maxiter;      /* iterations (Arnoldi columns) before the fallback      */
  int smooth;           /* damped-Jacobi sweeps after the network (0..32)        */
  double omega;         /* their damping                                         */
  int check_every;      /* iterations between host checks of the residual        */
  int stall_checks;     /* fallback when the best ||r|| has not fallen by         */
  double stall_factor;  /* stall_factor within stall_checks x check_every iters  */
                        /* (flexible GMRES: checked after each restart cycle on  */
                        /* the true residual, same window in Arnoldi columns)    */
  int fallback;         /* 1: finish with plain Jacobi PCG after a stall          */
  int use_graph;        /* 1: replay one iteration as a CUDA graph                */
  int window;           /* stored directions of the truncated flexible CG (1..8) */
  int outer;            /* outer method: 0 flexible CG, 1 flexible GMRES          */
  int restart;          /* flexible GMRES restart length (1..128)                 */
} tpf_learned_options;

typedef struct tpf_lppe_result {
  int64_t iterations;           /* flexible-CG / -GMRES iterations (network applications) */
  int64_t fallback_iterations;  /* plain PCG iterations after a stall             */
  int64_t restarts;             /* restarts from the true residual                */
  double rel_residual;          /* ||b - S p|| / ||b|| at exit                     */
  int info;                     /* 0 converged                                     */
  int fell_back;                /* 1 when the plain PCG fallback ran               */
} tpf_lppe_result;

typedef struct tpf_lppe tpf_lppe;

void tpf_lppe_default_options(tpf_learned_options* opts);
/* Learned solver on a 2-D PPE handle.  coarsen = 1: the network reads the
 * fine residual (image = node counts rounded up to multiples of 8);
 * coarsen = b in {2, 4, 8}: two-level mode, the network solves the problem
 * aggregated over b x b node blocks (image = ceil(n / b) rounded up to 8)
 * inside a V(1, smooth) cycle with damped-Jacobi sweeps on the fine grid. */
int tpf_lppe_create(tpf_lppe** lp, tpf_ppe* ppe, tpf_unet* net, int coarsen);
int tpf_lppe_destroy(tpf_lppe* lp);
/* tpf_ppe_prepare plus the density feature of the network input. */
int tpf_lppe_prepare(tpf_lppe* lp, const double* rho, void* stream);
/* Same contract as tpf_ppe_solve (p[pin] = 0, TPF_ENOCONV when the budget
 * ends), flexible CG (outer = 0) or flexible GMRES(restart) (outer = 1)
 * preconditioned by the network; after a stall or at the end of the budget
 * plain Jacobi PCG finishes from the current iterate when fallback = 1. */
int tpf_lppe_solve(tpf_lppe* lp, const double* rhs, const double* rho, double* p, const double* p_init,
                   const tpf_learned_options* opts, void* stream, tpf_lppe_result* result);
/* z = B(r), the preconditioner alone (r, z device vectors of the grid). */
int tpf_lppe_precondition(tpf_lppe* lp, const double* r, double* z, int smooth, double omega, void* stream);
/* Damped-Jacobi sweeps per smoother launch, 1..4 (default 4): the blocked
 * smoother keeps a tile and a halo as wide as its sweeps in shared memory;
 * every setting gives the same bits. */
int tpf_lppe_set_smooth_block(tpf_lppe* lp, int sweeps);
/* zout = J^sweeps(zin): damped-Jacobi sweeps z + omega D^-1 (r - S z) (pin
 * 0) of the prepared operator, the preconditioner's smoother alone (zin, r,
 * zout device vectors of the grid; zout may alias zin). */
int tpf_lppe_smooth(tpf_lppe* lp, const double* zin, const double* r, double* zout, int sweeps, double omega,
                    void* stream);
/* Training pair from an error field e of the weighted system (pin 0), in the
 * form the network reads (in2, target: device FP32 on the network image).
 * coarsen = 1: in2 = (D^-1/2 S e / s, density feature, couplings of
 * D^-1/2 S D^-1/2 to the next row / column), target = D^1/2 e / s
 * (s = rms of D^-1/2 S e).  Two-level mode: with r = S e, the pre-smoothing
 * sweep z1 = omega D^-1 r, r1 = r - S z1 and e1 = e - z1,
 * in2 = (D_c^-1/2 R r1 / s_c, aggregate density feature, scaled Galerkin
 * couplings to the next row / column) and
 * target = D_c^1/2 mean_aggregate(e1) / s_c. */
int tpf_lppe_pair(tpf_lppe* lp, const double* e, float* in2, float* target, double omega, void* stream);
/* Two-level mode: the data of the energy loss for an error field e: in2 as
 * tpf_lppe_pair, coupl [H][W][2] = scaled Galerkin couplings of the coarse
 * operator, *escale (device) = (e1 . S e1) / s_c^2. */
int tpf_lppe_pair_energy(tpf_lppe* lp, const double* e, float* in2, float* coupl, double* escale, double omega,
                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TPF_H_ */
