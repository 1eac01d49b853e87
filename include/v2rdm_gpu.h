/*
 * v2rdm_gpu.h -- C ABI of the B200 boundary-point SDP solver for the
 * active-space hot path of v2RDM-CASSCF.
 *
 * The plugin's solver object (v2RDMSolver, v2rdm_solver.h:79-575) keeps the
 * BPSDP state in Psi4 vectors and runs the outer loop of compute_energy
 * (v2rdm_solver.cc:1778-1908) on the host.  These entry points replace that
 * loop and the functions it calls:
 *
 *   v2g_create                 common_init's layout part (v2rdm_solver.cc:487-1285)
 *                              and BuildBasis (basis.cc:439-757)
 *   v2g_set_hamiltonian        GetIntegrals/RepackIntegrals/FrozenCoreEnergy
 *                              (tei.cc:55-313) for DF/CD three-index integrals
 *   v2g_guess_random           Guess, TPDM_GUESS=RANDOM (v2rdm_solver.cc:2479-2490)
 *   v2g_set_state/get_state    the x, y, z, mu members; checkpoint restart
 *                              (checkpoint.cc:56-121)
 *   v2g_apply_A / v2g_apply_AT bpsdp_Au / bpsdp_ATu (v2rdm_solver.cc:3020-3158)
 *   v2g_solve                  the outer loop (v2rdm_solver.cc:1778-1908) with
 *                              CGSolver::solve (cg_solver.cc:125-177) and
 *                              Update_xz (v2rdm_solver.cc:3216-3289)
 *   v2g_solve_batch            many such solves in one lock-step GPU run
 *
 * Conventions: every function returns V2G_OK (0) or a negative status; no
 * C++ exception crosses this boundary.  v2g_last_error() gives the message of
 * the last failure on the calling thread.  All arrays are host memory in the
 * reference's layout (x, z: dimx; y, b: nconstraints), except the *_device
 * entry points, which take device pointers on the handle's stream.  A handle
 * is used by one host thread at a time.
 */
#ifndef V2RDM_GPU_H
#define V2RDM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define V2G_OK 0
#define V2G_ERR_ARG -1          /* invalid argument or option value */
#define V2G_ERR_CUDA -2         /* CUDA runtime failure */
#define V2G_ERR_NOT_CONVERGED -3 /* MAXITER reached ("v2RDM did not converge.") */
#define V2G_ERR_NONFINITE -4    /* NaN or Inf appeared in the iteration */
#define V2G_ERR_UNSUPPORTED -5  /* option combination not built */
#define V2G_ERR_NO_DEVICE -6    /* no CUDA device visible */

typedef struct v2g_handle v2g_handle;

/* Options on the hot path, same names and defaults as the plugin
 * (plugin.cc:66-124); fill with v2g_default_options(). */
typedef struct v2g_options {
    const char* positivity;     /* "D", "DQ", "DG", "DQG", "DQGT1", "DQGT2", "DQGT1T2" */
    int constrain_spin;         /* CONSTRAIN_SPIN (1) */
    int constrain_sz;           /* CONSTRAIN_SZ (1) */
    double r_convergence;       /* R_CONVERGENCE (1e-4) */
    double e_convergence;       /* E_CONVERGENCE (1e-4) */
    double cg_convergence;      /* CG_CONVERGENCE (1e-9) */
    int maxiter;                /* MAXITER (10000) */
    int cg_maxiter;             /* CG_MAXITER (10000) */
    double tau_parameter;       /* TAU_PARAMETER (1.0) */
    int mu_update_frequency;    /* MU_UPDATE_FREQUENCY (500) */
    int device;                 /* CUDA device ordinal (0) */
    int record_trace;           /* keep the per-iteration line of v2rdm_solver.cc:1881 (0) */
    int profile;                /* time every A / A^T launch of the CG with CUDA events (0) */
    int adaptive_projection;    /* 1: Update_xz accepts an eigendecomposition whose off-diagonal
                                   residual is below 0.01 min(eps(p), eps(d)), the CG tolerance
                                   rule (x, z stay PSD); 0: every projection converged, as the
                                   plugin (0) */
    double cg_tolerance_factor; /* CG stops at factor * min(eps(p), eps(d)) after the first outer
                                   iteration; 0.01 is the plugin's rule (v2rdm_solver.cc:1797-1805),
                                   and values up to 0.1 trade fewer CG iterations for a few more
                                   outer ones (0.01) */
    int spin_adapt_q2;          /* SPIN_ADAPT_Q2 (plugin.cc): Q2 as singlet / triplet blocks (0) */
    int spin_adapt_g2;          /* SPIN_ADAPT_G2: G2 as singlet / triplet blocks; needs
                                   constrain_spin = 0, as the plugin's maximal spin constraint
                                   reads the unadapted G2ba block (0) */
    int constrain_d3;           /* CONSTRAIN_D3: 3-RDM positivity and its partial traces (0) */
    int constrain_d4;           /* CONSTRAIN_D4: 4-RDM positivity and its partial traces; implies
                                   constrain_d3, as in the plugin (0) */
    int start;                  /* 0: solve from the handle's state (v2g_guess_random, the plugin's
                                   TPDM_GUESS=RANDOM, or v2g_set_state); 1: from the least-norm
                                   point of A x = b with zero duals and mu = 1, computed on the
                                   GPU at the start of the solve; 2: from the learned warm start's
                                   proposal (v2g_ws_propose) moved onto A x = b the same way, with
                                   zero duals and the proposed mu, or as 1 without a proposal
                                   (1 and 2 have no counterpart in the plugin) (0) */
    int cg_extrapolate;         /* 1: each outer iteration's CG starts from y_k + (y_k - y_{k-1}),
                                   the linear extrapolation of the last two CG solutions, instead of
                                   y_k (cg_solver.cc:125 warm-starts from y_k); the stopping test is
                                   unchanged, so only the CG iteration count changes (0) */
    int anderson_memory;        /* m > 0: Anderson acceleration of the outer iteration: the next
                                   (x, z) is the step's result minus the combination of the last m
                                   step differences that minimises the fixed-point residual; the
                                   stopping test and the energies are taken on the un-accelerated
                                   step as in the plugin; the history restarts when mu changes;
                                   0 = off, at most 16 (0) */
    int mixed_precision;        /* 1: while an instance's adaptive projection tolerance (see
                                   adaptive_projection) is at least 1e-5, the dense products of the
                                   projection of its large blocks (refinement residuals, eigenvector
                                   updates, x = V D+ V^T and z = V D- V^T) run on the tensor cores as
                                   3xTF32 products with FP32 accumulation (FP32 accuracy); below it
                                   they run in FP64, whose first refinement sweeps take the
                                   eigenvectors from FP32 to FP64 accuracy.  Maps, CG, errors and
                                   energies stay FP64.  Needs adaptive_projection (0) */
} v2g_options;

typedef struct v2g_result {
    double e_total;      /* c.x + enuc + efzc ("v2RDM total energy") */
    double e_primal;     /* c.x + enuc + efzc at the last iteration */
    double e_dual;       /* b.y + enuc + efzc */
    double ep;           /* ||A x - b|| */
    double ed;           /* ||A^T y - c + z|| */
    double mu;
    double efzc, enuc;
    long oiter;          /* outer (macro) iterations */
    long iiter;          /* total CG (micro) iterations */
    int status;          /* V2G_OK, V2G_ERR_NOT_CONVERGED, V2G_ERR_NONFINITE */
    double t_cg;         /* device seconds in the CG phase (iiter_time_) */
    double t_xz;         /* device seconds in Update_xz (oiter_time_) */
    double t_total;      /* device seconds for the whole solve */
    long cg_stalls;      /* CG solves stopped because the residual grew 100x above its
                            minimum (a right-hand side with a component in the null space of
                            A^T above the CG tolerance; the plugin's CG would diverge there) */
} v2g_result;

void v2g_default_options(v2g_options* opt);
const char* v2g_last_error(void);

/* Active-space problem.  Orbital counts per irrep in Pitzer order, like the
 * plugin's frzcpi/rstcpi/active/rstvpi/frzvpi; nalpha/nbeta are total electron
 * counts of the reference wavefunction (the active counts are nalpha minus
 * the doubly occupied core).  multiplicity = 2S+1. */
int v2g_create(const v2g_options* opt, int nirrep, const int* frzcpi, const int* rstcpi, const int* amopi,
               const int* rstvpi, const int* frzvpi, int nalpha, int nbeta, int multiplicity, v2g_handle** out);
void v2g_destroy(v2g_handle* h);

/* Sizes: dimx_, nconstraints_, and the PSD blocks (dimensions_). */
long v2g_dimx(const v2g_handle* h);
long v2g_nconstraints(const v2g_handle* h);
int v2g_nblocks(const v2g_handle* h);
int v2g_block_dims(const v2g_handle* h, int* dims);

/* Integrals: oei packed per irrep as lower triangles over the orbitals that
 * are not frozen virtuals (oei_full_sym_), and three-index integrals
 * qmo[Q * ntri + INDEX(p,q)], ntri = nmo'(nmo'+1)/2 (Qmo_, tei.cc:321). */
int v2g_set_hamiltonian(v2g_handle* h, const double* oei_packed, const double* qmo, int nq, double enuc);
int v2g_get_c(const v2g_handle* h, double* c);
int v2g_get_b(const v2g_handle* h, double* b);
double v2g_efzc(const v2g_handle* h);

/* Starting point: the reference's random guess (srand(0), glibc rand) or an
 * explicit state (restart from a checkpoint, warm start). */
int v2g_guess_random(v2g_handle* h);
int v2g_set_state(v2g_handle* h, const double* x, const double* y, const double* z, double mu);
int v2g_get_state(const v2g_handle* h, double* x, double* y, double* z, double* mu);

/* Constraint maps on host vectors (copied through the device) and on device
 * vectors.  out = A u (length nconstraints) or A^T u (length dimx). */
int v2g_apply_A(v2g_handle* h, const double* u, double* out);
int v2g_apply_AT(v2g_handle* h, const double* u, double* out);
int v2g_apply_A_device(v2g_handle* h, const double* d_u, double* d_out);
int v2g_apply_AT_device(v2g_handle* h, const double* d_u, double* d_out);

/* The maps applied to nvec vectors at once, stored instance-interleaved on
 * the device (element e of vector v at [e * nvec + v], 1 <= nvec <= 256), on
 * the given CUDA stream (NULL: the legacy default stream).  Asynchronous. */
int v2g_apply_A_batched_device(v2g_handle* h, int nvec, const double* d_u, double* d_out, void* stream);
int v2g_apply_AT_batched_device(v2g_handle* h, int nvec, const double* d_u, double* d_out, void* stream);

/* One projection step on the handle's state, as Update_xz: with
 * U = A^T y - c + mu x per block, x = U+/mu and z = -U-. */
int v2g_update_xz(v2g_handle* h, double mu);

/* The projection step of v2g_update_xz on caller-owned device vectors,
 * allocating no device memory.  No counterpart in the reference: it is for
 * host programs that cannot call cudaMalloc while they run (a pool allocator
 * that owns all device memory, a fixed device-memory budget).  Device memory
 * in: d_c (dimx doubles) and d_y (nconstraints doubles); in/out: d_x (dimx);
 * out: d_z (dimx).  Limits: every block of dimension <= 64 and dimx <= 65536,
 * else V2G_ERR_ARG; the handle's device tables must exist (v2g_update_xz, a
 * map call or a solve builds them).  Scratch is a static device array of
 * about 0.5 MiB that every GPU loading the library holds until exit; the
 * first call on a device looks up its address, so make that call before any
 * stream capture.  mu and the block list reach the device as a kernel
 * argument: no host memory is copied.  Calls share the array: calls that
 * overlap on the GPU (other streams or host threads) race.  Asynchronous on
 * the given stream (NULL: the legacy default stream); the caller's current
 * device is left as it was. */
int v2g_update_xz_noalloc(v2g_handle* h, double mu, const double* d_c, const double* d_y, double* d_x, double* d_z,
                          void* stream);

/* Seconds per launch of A and of A^T (the map kernels of the CG) on nvec
 * instance-interleaved vectors of the handle's layout: `reps` launches
 * captured in a CUDA graph and replayed between CUDA events on one stream, so
 * the figure is the kernels' own duration (plus the graph's launch gaps), not
 * the host's launch rate; every kernel variant is timed and the fastest
 * reported, as the solver's autotuner picks it.  For roofline figures; no
 * counterpart in the reference. */
int v2g_time_maps(v2g_handle* h, int nvec, int reps, double* sec_A, double* sec_AT);

/* The dense product of the projection on caller-owned device buffers, for
 * tests and inspection: for nblocks symmetric blocks of dimensions dims[i]
 * (each padded to np_i = dims rounded up to a multiple of 64 and stored
 * row-major np_i x np_i, one after the other), C_i = op(A_i) diag(d_i) op(B_i)
 * with op = transpose where trans* is set and d (np_i per block, one after the
 * other) optional.  tensor_cores = 1 runs the 3xTF32 tcgen05 kernel of the
 * mixed-precision projection, 0 the FP64 kernel.  Synchronous; returns
 * V2G_ERR_CUDA when a tensor-core pipeline wait ran out.  No counterpart in
 * the reference (it calls F_DGEMM, v2rdm_solver.cc:3273,3286). */
int v2g_block_gemm_device(int nblocks, const int* dims, const double* A, int transA, const double* B, int transB,
                          const double* d, double* C, int tensor_cores, int device);

/* Seconds per product C_i = A_i B_i of v2g_block_gemm_device (no transposes, no
 * scaling) on caller-owned device buffers: 3 warm-up products, then `reps`
 * back to back on one stream between CUDA events.  With tensor_cores = 1 a
 * product is the two TF32 split launches and the tcgen05 MMA launch.  For
 * roofline figures; no counterpart in the reference. */
int v2g_time_block_gemm(int nblocks, const int* dims, const double* A, const double* B, double* C, int tensor_cores,
                        int reps, int device, double* sec);

/* Learned warm start (no counterpart in the reference, whose start is the
 * random guess of Guess, v2rdm_solver.cc:2386-2516).  A pair-wise MLP (16
 * features of each orbital pair p <= q from h and the three-index integrals,
 * three hidden ReLU layers of width `hidden`, BF16 weights, FP32 arithmetic)
 * proposes for every pair the alpha 1-RDM element gamma_pq, the D2ab pair
 * diagonal D2ab(pq,pq) and a contribution to log(mu).  It is trained on the
 * GPU (Adam on the mean squared error) on converged solutions of this solver;
 * v2g_ws_propose turns its output into the handle's start proposal x0 (D1,
 * Q1 = 1 - D1, the D2ab diagonal; zero elsewhere) and mu, which a solve with
 * start = 2 projects onto A x = b.  All-active C1 singlets only
 * (V2G_ERR_UNSUPPORTED otherwise).  Rows are the n (n + 1) / 2 pairs of an
 * active space, features 16 floats per row, targets and outputs 3. */
typedef struct v2g_warmstart v2g_warmstart;
int v2g_ws_create(int hidden, int device, unsigned long long seed, v2g_warmstart** out);
void v2g_ws_destroy(v2g_warmstart* w);
long v2g_ws_num_params(const v2g_warmstart* w);
int v2g_ws_get_params(const v2g_warmstart* w, float* params);   /* FP32 master weights */
int v2g_ws_set_params(v2g_warmstart* w, const float* params);   /* also resets the optimiser */
long v2g_ws_rows(const v2g_handle* h);                             /* pairs of the handle's active space */
int v2g_ws_features(const v2g_handle* h, float* features);          /* rows x 16 */
int v2g_ws_targets(const v2g_handle* h, float* targets);            /* rows x 3 from the handle's x and mu */
int v2g_ws_forward(v2g_warmstart* w, long rows, const float* features, float* out);
/* loss = mean squared error over rows x 3 outputs and its gradient (FP32,
 * num_params floats, laid out like the parameters) */
int v2g_ws_gradient(v2g_warmstart* w, long rows, const float* features, const float* targets, double* loss,
                    float* grad);
/* Adam (lr) over minibatches of batch_rows rows in the given order, `epochs`
 * passes; loss = the last epoch's mean */
int v2g_ws_train(v2g_warmstart* w, long rows, const float* features, const float* targets, int epochs,
                 int batch_rows, float lr, double* loss);
/* use_mu = 1: the proposed mu; 0: mu = 1 with the proposed primal */
int v2g_ws_propose(v2g_warmstart* w, v2g_handle* h, int use_mu);

/* The RDMs handed to the orbital optimiser, as PackSpatialDensity
 * (v2rdm_solver.cc:3664-3773), from the handle's x: d1 = spin-summed 1-RDM,
 * per irrep, packed lower triangle (d1_act_spatial_sym_); d2 = spin-free
 * 2-RDM over spatial pairs, per irrep, packed lower triangle
 * (d2_act_spatial_sym_).  active_energies (Pitzer order, one per active
 * orbital) fix the numbering of the spatial pairs as the plugin's orbital
 * energies do (basis.cc:626-652); NULL numbers them in Pitzer order.  The
 * values equal the reference's bit for bit. */
int v2g_spatial_density_dims(const v2g_handle* h, long* d1_dim, long* d2_dim);

/* Orbital energies of the active orbitals (Pitzer order), as the plugin's
 * epsilon_a_: they number the spatial pairs of the spin-adapted Q2 singlet
 * block and of the packed 2-RDM (basis.cc:626-652).  Without this call the
 * pairs follow Pitzer order, which is the reference's for C1.  Call before the
 * first map or solve of the handle (its device tables are rebuilt). */
int v2g_set_active_orbital_energies(v2g_handle* h, const double* energies);
int v2g_pack_spatial_density(v2g_handle* h, const double* active_energies, double* d1, double* d2);

/* Checkpoint and restart (WriteCheckpointFile / ReadFromCheckpointFile,
 * checkpoint.cc:56-121): the entries MU, PRIMAL, DUAL 1, DUAL 2 of the
 * handle's state in a small named-record file (not Psi4's PSIO container).
 * Reading checks that the file belongs to the same layout. */
int v2g_write_checkpoint(const v2g_handle* h, const char* path);
int v2g_read_checkpoint(v2g_handle* h, const char* path);

/* The full BPSDP solve from the handle's current state. */
int v2g_solve(v2g_handle* h, v2g_result* res);

/* One-step orbital optimisation runs the BPSDP loop with RotateOrbitals (focas)
 * every ORBOPT_FREQUENCY outer iterations inside it (v2rdm_solver.cc:1855-1873):
 * mu, the outer-iteration count (the mu schedule), the last eps(p) / eps(d)
 * (the next CG tolerance) and x, y, z carry on across the rotations.  This
 * continues the handle's loop where the previous v2g_solve / v2g_solve_continue
 * stopped, for at most max_outer outer iterations, so the caller can rotate the
 * orbitals and call v2g_set_hamiltonian between segments.  Returns
 * V2G_ERR_NOT_CONVERGED when the segment ended unconverged (res->oiter counts
 * from the start of the loop; res->iiter counts this segment). */
int v2g_solve_continue(v2g_handle* h, int max_outer, v2g_result* res);

/* Solves count independent problems in one GPU run.  Handles with the same
 * layout share index tables; each keeps its own convergence test and stops
 * independently.  Returns V2G_OK when every instance converged. */
int v2g_solve_batch(v2g_handle** hs, int count, v2g_result* res);

/* Timing of the last v2g_solve / v2g_solve_batch call on this thread.
 * device_seconds covers the solve with inputs already on the device (CUDA
 * events around the iteration phase); e2e_seconds covers the whole call,
 * host-to-device copies of x, y, z, c and device-to-host copies of the results
 * included.  map_* are filled when the handles were created with profile=1:
 * summed CUDA-event durations of the A and A^T launches inside CG, their count
 * and their algorithmic bytes (8 * (rows + columns) per instance). */
typedef struct v2g_batch_stats {
    double device_seconds;
    double e2e_seconds;
    long kernel_launches;     /* kernels issued by this library during the solve */
    double map_seconds;
    long map_launches;
    double map_bytes;
    long groups;              /* layouts solved concurrently */
    double h2d_bytes, d2h_bytes;
    long refine_sweeps;       /* Ogita-Aishima sweeps over the large PSD blocks */
    long jacobi_sweeps;       /* block-Jacobi sweeps (cold starts and fallbacks) */
    long jacobi_blocks;       /* large blocks that fell back to block Jacobi */
    long jacobi_unconverged;  /* of those, blocks whose refinement was still short of its
                                 tolerance after its sweep cap (the others had a first-order
                                 step too large to trust) */
} v2g_batch_stats;
int v2g_last_batch_stats(v2g_batch_stats* out);

/* The constraint matrix A (nconstraints x dimx) as CSR, built on the host;
 * no GPU needed.  v2g_A_nnz gives the entry count; v2g_export_A fills
 * rowptr (nconstraints + 1), col and val (nnz each).  These expose the
 * operator that bpsdp_Au applies (v2rdm_solver.cc:3020-3065) for inspection
 * and for integrations that apply it themselves. */
long v2g_A_nnz(v2g_handle* h);
int v2g_export_A(v2g_handle* h, long* rowptr, int* col, double* val);

/* Per-iteration trace (oiter, iiter, E(p), E(d), gap, mu, eps(p), eps(d)) of
 * the last solve when record_trace was set; returns the number of rows. */
long v2g_trace(const v2g_handle* h, double* rows, long cap);

#ifdef __cplusplus
}
#endif

#endif /* V2RDM_GPU_H */
