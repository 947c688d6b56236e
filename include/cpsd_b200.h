/*
 * cpsd_b200.h -- C ABI of the B200 (sm_100a) steepest-descent engine.
 *
 * Drop-in for the serial Simple-CPSD electronic minimisation
 * (Cpsd-mpi-bamboo/ccpsdv3): a program that linked cpsd.o and the FFTPACK
 * 3-D wrapper links this library instead and runs the same loop on the GPU.
 * All pointers are host pointers in the reference's layouts (half box of
 * (nfft/2+1) x nfft x nfft complex per band = n2ft3d doubles; real-space
 * arrays padded to (nfft+2) x nfft x nfft).  Supported grids: nfft in
 * {16, 24, 32, 48, 64, 128}; bands per spin <= 256.  There is no CPU
 * fallback: without a usable GPU every call fails.
 */
#ifndef CPSD_B200_H
#define CPSD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    CPSD_OK = 0,
    CPSD_ERR_CUDA = 1,          /* a CUDA call failed (no device, out of memory, ...) */
    CPSD_ERR_ARG = 2,           /* an argument is out of range or inconsistent */
    CPSD_ERR_GRID = 3,          /* nfft not one of the supported sizes */
    CPSD_ERR_BANDS = 4,         /* more than 256 bands in a spin channel */
    CPSD_ERR_EMPTY_MASK = 5,    /* the cutoff mask selects no G vector */
    CPSD_ERR_UNMASKED_PSI = 6,  /* input orbitals have coefficients outside the mask */
    CPSD_ERR_MOVE = 7,          /* move=1 requested but no G vectors / masses were given */
    CPSD_ERR_TIMEOUT = 8,       /* a bounded wait on the device ran out (tensor-core pipeline) */
    CPSD_ERR_SCRATCH = 9,       /* a problem larger than cpsd_overlap_tn_noalloc's static scratch */
    CPSD_WARN_LAGRANGE = 10,    /* (positive warning) Lagrange iteration hit 30 steps; the
                                   reference prints "ierr=10" and continues (cpsd.c:477) */
    CPSD_ERR_EIG = 11,          /* the epilogue's eigen solve of hml did not converge */
    CPSD_ERR_IO = 12            /* an output file could not be written */
};

/* Human-readable text for a status code. */
const char *cpsd_gpu_strerror(int status);

/* ------------------------------------------------------ drop-in entry points */

/*
 * Replaces void cpsd(...) of ccpsdv3/cpsd.c:33-71 (prototype repeated at
 * ccpsdv3/main.c:18-56), same arguments and meanings: runs `inner`
 * steepest-descent steps from c2, then the energies E[0..9] and the
 * convergence measures.  On exit c1 holds the orbitals of the last step, c2
 * the next iterate, cpsi = c2 - c1, dn the spin densities of the last step,
 * hml/lmd the Hamiltonian and Lagrange matrices.  cpsdwork is accepted and
 * not used (scratch lives on the GPU).  Errors are printed like the
 * reference's and the call returns; use cpsd_gpu_cpsd() for a status.
 *
 * The library keeps one device context per shape (grid, bands, ions, kinds,
 * mask).  A call of the same shape as the last one starts its steps on the
 * mask and tables the context holds and compares them with the ones passed
 * (and c2 with zero outside the mask) on host threads meanwhile; if
 * anything differs the steps are discarded and the call runs again on the
 * new inputs, so the outputs are always those of the inputs passed.  c2
 * with values outside the mask is refused (CPSD_ERR_UNMASKED_PSI) with
 * every output left untouched.
 */
void cpsd(const int inner, const int move, const int nion, const int ispin, const int *ne,
          const int nfft, const int nfft3d, const int n2ft3d, const double *unitg,
          const double omega, const double dt, const double fmass, const int *katm,
          const double *amass, const double *zv, const int nsh, const double *rcell,
          const double cewald, const double rcut, const int *masker, const double *G,
          const double *tg, const double *vc, const double *vg, int *lmmax, double *vnlnrm,
          double *vl, double *vnl, double *r1, double *r2, double *fion, double *c1, double *c2,
          double *cpsi, double *dn, double *hml, double *lmd, double *cpsdwork, double *E,
          double *deltae, double *deltac, double *deltar);

/* cpsd() returning a status (CPSD_OK, an error, or CPSD_WARN_LAGRANGE). */
int cpsd_gpu_cpsd(const int inner, const int move, const int nion, const int ispin, const int *ne,
                  const int nfft, const int nfft3d, const int n2ft3d, const double *unitg,
                  const double omega, const double dt, const double fmass, const int *katm,
                  const double *amass, const double *zv, const int nsh, const double *rcell,
                  const double cewald, const double rcut, const int *masker, const double *G,
                  const double *tg, const double *vc, const double *vg, const int *lmmax,
                  const double *vnlnrm, const double *vl, const double *vnl, double *r1, double *r2,
                  double *fion, double *c1, double *c2, double *cpsi, double *dn, double *hml,
                  double *lmd, double *E, double *deltae, double *deltac, double *deltar);

/*
 * Replace the Fortran-ABI cr_fft3b / rc_fft3f of fftpack3d/fftpack3d.f:22-96
 * and :107-196 (called from ccpsdv3/cpsd.c:179,201,380,390): in-place,
 * unnormalised complex->real inverse and real->complex forward 3-D FFTs of
 * one (nx+2) x ny x nz array.  Only cubic nx = ny = nz with the reference's
 * strides (inc2c = nx/2+1, inc3c = (nx/2+1)*ny, inc2r = nx+2, inc3r =
 * (nx+2)*ny) are accepted; tmp/ntmp are ignored.  The whole box is
 * transformed (no sphere pruning).
 */
void cr_fft3b_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r, int *nx, int *ny,
               int *nz, double *tmp, int *ntmp);
void rc_fft3f_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r, int *nx, int *ny,
               int *nz, double *tmp, int *ntmp);

/* Status of the last cr_fft3b_/rc_fft3f_ call on this thread. */
int cpsd_gpu_fft_status(void);

/* ------------------------------------------------------ persistent context */

typedef struct cpsd_gpu_ctx cpsd_gpu_ctx;

enum { CPSD_PREC_FP64 = 0, CPSD_PREC_MIXED = 1 };
/* Engine of the TN products of the mixed path: FP64 CUDA cores, or three
 * TF32 tensor-core products (hi*hi + hi*lo + lo*hi, FP32 accumulate in tensor
 * memory, FP64 split-K sums), about FP32 accuracy.  CPSD_GEMM_TF32X3 moves
 * the KB projector contraction and back-projection (and the learned step's
 * residual) to the tensor cores; CPSD_GEMM_TF32X3_OVERLAPS moves the three
 * Lagrange overlaps and the constraint correction as well.  The
 * Lagrange solve divides (1 - <c2|c2>) by dte (about 1e-2), so FP32-level
 * overlaps cost about 1e-6 relative in the energy per step: follow such a
 * run with FP64 steps. */
enum { CPSD_GEMM_FP64 = 0, CPSD_GEMM_TF32X3 = 1, CPSD_GEMM_TF32X3_OVERLAPS = 3 };

typedef struct {
    int nfft;        /* grid edge */
    int ispin;       /* 1 or 2 */
    int ne[2];       /* bands per spin */
    int nion;        /* ions */
    int nkatm;       /* ion kinds */
    int nsh;         /* real-space Ewald image cells (27 in the reference) */
    int precision;   /* CPSD_PREC_FP64 (parity path) or CPSD_PREC_MIXED */
    int device;      /* CUDA device ordinal */
    double unitg[9]; /* reciprocal lattice, ccpsdv3/get_cube.c */
    double omega, dt, fmass, cewald, rcut;
} cpsd_gpu_params;

/*
 * Create a context for one cell.  masker1 is the nfft3d-long cutoff mask of
 * ccpsdv3/get_masker.c (one int per half-box G, not the duplicated
 * n2ft3d-long array cpsd() takes).  All GPU memory is allocated here.
 */
int cpsd_gpu_create(const cpsd_gpu_params *p, const int *masker1, cpsd_gpu_ctx **out);

/* Change the per-call scalars cpsd() receives (lattice, volume, time step,
 * fictitious mass, Ewald constant and cut radius) without rebuilding. */
int cpsd_gpu_set_scalars(cpsd_gpu_ctx *c, const double *unitg, double omega, double dt, double fmass,
                         double cewald, double rcut);

/* Upload the per-cell tables in the layouts cpsd() takes.  G (3 x nfft3d,
 * ccpsdv3/get_g.c) and amass (per kind) are needed only for move = 1 and may
 * be NULL otherwise. */
int cpsd_gpu_set_tables(cpsd_gpu_ctx *c, const int *katm, const double *amass, const double *zv,
                        const double *rcell, const double *G, const double *tg, const double *vc,
                        const double *vg, const int *lmmax, const double *vnlnrm, const double *vl,
                        const double *vnl);

/* Upload orbitals (half box, (ne0+ne1) x n2ft3d doubles) and ion positions. */
int cpsd_gpu_set_state(cpsd_gpu_ctx *c, const double *c2, const double *r2);

/*
 * Run `inner` SD steps and the energy evaluation, the body of cpsd().
 * E[0] must hold the previous total energy (for deltae), as in cpsd().
 * move = 1 also computes the ion forces (local, nonlocal, k- and real-space
 * Ewald, cpsd.c:246-364) and takes the ion step r2 = r1 + dt/sqrt(M) fion
 * (cpsd.c:401-411); deltar is then the largest |fion| of the last step.
 */
int cpsd_gpu_run(cpsd_gpu_ctx *c, int inner, int move, double *E, double *deltae, double *deltac,
                 double *deltar);

/* Download the state cpsd() returns; any pointer may be NULL to skip it.
 * c1, c2 and cpsi are written on host threads in parallel (zeros, then the
 * sphere's coefficients): they must be distinct, non-overlapping arrays, as
 * the reference's driver allocates them (main.c:126-136). */
int cpsd_gpu_get_state(cpsd_gpu_ctx *c, double *c1, double *c2, double *cpsi, double *dn,
                       double *hml, double *lmd, double *r1, double *r2, double *fion);

/*
 * The run's epilogue, ccpsdv3/main.c:452-487, on the resident state after at
 * least one cpsd_gpu_run (CPSD_ERR_ARG before).  Any output may be NULL:
 *   ortho  <c1_i|c1_j> per spin (Gamma-point dots), hml's layout: the
 *          orthonormality table main.c:455-467 prints for i <= j;
 *   eig    eigenvalues of hml per spin, eig[ms*ne[0] + i], descending: what
 *          esyev('V','U') + eigsrt leave (main.c:470-479);
 *   vec    the eigenvectors, hml's layout, columns in eig's order (the hml
 *          that main.c holds after esyev + eigsrt); a column's sign is not
 *          fixed by the problem and may differ from LAPACK's.
 * Then c1 <- c2 vec per spin on the device (main.c:481-487): a following
 * cpsd_gpu_get_state returns the rotated orbitals main.c writes to ELCOUT.
 * CPSD_ERR_EIG: the Jacobi solve did not converge (not seen in practice).
 */
int cpsd_gpu_epilogue(cpsd_gpu_ctx *c, double *ortho, double *eig, double *vec);

/*
 * ELCOUT as main.c:537-546 writes it: int icube, int nfft, double unit,
 * int ispin, int ne[2], then (ne[0]+ne[1]) * (nfft+2)*nfft*nfft doubles of
 * c1 (host layout), native byte order.  CPSD_ERR_IO if the file cannot be
 * written.
 */
int cpsd_write_elcout(const char *path, int icube, int nfft, double unit, int ispin, const int *ne,
                      const double *c1);

/*
 * IONOUT as main.c:549-566 writes it: nkatm; per kind "'<fname> ' <lmax>";
 * nion; per ion "<katm+1> x y z 0.000000 0.000000 0.000000 " -- main.c
 * zeroes r1 (:550) before printing it beside r2.  fname[ia] are the psp file
 * names IONIN listed.
 */
int cpsd_write_ionout(const char *path, int nkatm, const char *const *fname, const int *lmax, int nion,
                      const int *katm, const double *r2);

/*
 * Input pipeline.  Replaces kbpp() of ckbppv3/dkbppv3.c (kbppv3.c:335-444),
 * same arguments and meanings: Kleinman-Bylander tables on the half-box G
 * grid (G as get_g lays it out, 3 * nfft3d) from tabulated radial data --
 * rho[nrho] on a uniform grid of step drho, vp and wp [(lmax+1) * nrho],
 * channel lmax the local one.  As kbpp() does, vp's nonlocal channels are
 * replaced by vp_l - vp_lmax.  Out: vl[nfft3d], vnl[lmax^2 * nfft3d],
 * vnlnrm[lmax^2].  The per-G integrals run on the GPU (one thread per G;
 * the tables in shared memory), lmax <= 3, nrho <= 4095.
 */
int cpsd_gpu_kbpp(double zv, int lmax, int nrho, double drho, const double *rho, double *vp, const double *wp,
                  int nfft3d, const double *G, double *vl, double *vnl, double *vnlnrm);

/*
 * The initial orbitals of cmakepsi/dmakepsi.c:93-140: one plane wave per
 * band from PSI0.DAT rows (waves[4n..4n+3] = i j k l; coefficient 1, 1/sqrt(2)
 * or i/sqrt(2) for l = 0, > 0, < 0; on the kx = 0 plane also the Hermitian
 * partner), written into psi[(ne[0] + ne[1]) * (nfft+2)*nfft*nfft] in the
 * ELCIN layout; spin 1 reuses the first ne[1] rows, as the reference does.
 * Host code (a few stores per band); cpsd_write_elcout writes the file.
 * CPSD_ERR_ARG for an index outside the half box.
 */
int cpsd_makepsi(int nfft, int ispin, const int *ne, const int *waves, double *psi);

/* Sphere size (packed G vectors per band) and the kernel launches of one SD step. */
int cpsd_gpu_npw(const cpsd_gpu_ctx *c);
int cpsd_gpu_launches_per_step(const cpsd_gpu_ctx *c);
/* out[6]: npw, padded npw, (kx,ky) columns of the sphere, kx lines (KX),
 * KB projectors, density band chunks. */
int cpsd_gpu_geometry(const cpsd_gpu_ctx *c, int *out);
/* Steps whose Lagrange iteration stopped at 30 iterations, since creation. */
int cpsd_gpu_lagrange_failures(cpsd_gpu_ctx *c);

/* Cumulative counters: out[0] kernel launches, out[1] host-to-device bytes,
 * out[2] device-to-host bytes since the context was created. */
void cpsd_gpu_counters(const cpsd_gpu_ctx *c, long long *out);

/* Switch the transforms of the next steps between FP64 (the parity path)
 * and FP32 (mixed).  A context created with CPSD_PREC_MIXED holds both, so
 * the last steps can run as an FP64 refinement sweep on the same state; one
 * created with CPSD_PREC_FP64 accepts only CPSD_PREC_FP64. */
int cpsd_gpu_set_precision(cpsd_gpu_ctx *c, int precision);

/* SD steps are replayed from captured CUDA graphs unless switched off here
 * (or with the environment variable CPSD_B200_NO_GRAPHS set at creation). */
int cpsd_gpu_use_graphs(cpsd_gpu_ctx *c, int on);

/* Phase timing: with it on, CUDA events are recorded between the phases of
 * every SD step (inside the step graphs); cpsd_gpu_phase_times() returns the
 * durations (ms) of the phases of the last step and their count. */
int cpsd_gpu_phase_timing(cpsd_gpu_ctx *c, int on);
int cpsd_gpu_phase_times(cpsd_gpu_ctx *c, float *ms, int max);
const char *cpsd_gpu_phase_name(int i);

/* The context the drop-in cpsd() keeps between calls (NULL before the first
 * call).  The pointer stays valid only until the next cpsd() call whose
 * arguments describe a different cell (grid, bands, ions or precision), which
 * destroys that context and builds a new one; do not use it while another
 * thread is inside cpsd(). */
cpsd_gpu_ctx *cpsd_gpu_dropin_context(void);

/* ------------------------------------------------------ band-parallel SD
 * One cell stepped by several ranks (one GPU each), every rank holding the
 * whole state.  No counterpart in the serial reference; its MPI build
 * (ccpsdv3-mpi) splits the FFT grid instead (d3db-mpi.c:817-1099, the
 * reductions of Parallel.c:50-70 used at ccpsdv3-mpi/cpsd.c:385, 459-462).
 * Here the bands are split: rank r transforms, densifies and steps bands
 * [lo, hi) (phases 0 and 1), the caller sums the spin densities over the
 * ranks between phases 0 and 1 and gathers every rank's rows of c2 between
 * phases 1 and 2, and phase 2 (overlaps, Lagrange iteration, constraint,
 * cpsd.c:415-488) runs on all bands on every rank.  The caller's exchange
 * (an NCCL all-reduce and broadcasts over torch.distributed in
 * cpsd_b200.bands) runs on the context's stream, between the calls. */

/* Make the context step bands [lo, hi) only (hi < 0: every band again, the
 * ordinary path).  Not with a learned preconditioner or ion motion
 * (CPSD_ERR_ARG).  cpsd_gpu_run is refused while it is set. */
int cpsd_gpu_set_band_range(cpsd_gpu_ctx *c, int lo, int hi);
/* Enqueue phase 0, 1 or 2 of an SD step on the context's stream (without a
 * band range the three phases back to back are one ordinary SD step). */
int cpsd_gpu_step_phase(cpsd_gpu_ctx *c, int phase);
/* Device arrays of the exchanges: dn_part (this rank's spin densities,
 * ispin * nfft^3 doubles, after phase 0), dn (their sum, which the caller
 * writes before phase 1), c2 and cpsi (the current step's new orbitals and
 * -H psi, bands x ld doubles; after phase 1 rows [lo, hi) are this rank's). */
int cpsd_gpu_bp_buffers(cpsd_gpu_ctx *c, double **dn_part, double **dn, double **c2, double **cpsi, long *ld);
/* The energies of a call of `inner` band-parallel steps (cpsd.c:494-672),
 * after the caller has gathered every rank's rows of cpsi of the last step;
 * E[0] in: the previous total energy.  Every rank computes the same values. */
int cpsd_gpu_bp_finish(cpsd_gpu_ctx *c, int inner, double *E, double *deltae, double *deltac);

/* ------------------------------------------------------ tuning
 * Kernel choices of a context that change speed, not the algorithm (results
 * agree to rounding).  No counterpart in the reference.  The choices apply to
 * the transforms of the precision the context runs at the time of the call;
 * set them before batching the context (cpsd_gpu_batch_create). */
typedef struct {
    int plane_occupancy[4]; /* per plane pass (0 density, 1 V psi, 2 potential to r,
                               3 density to G): 0 = the build for one CTA per SM (up to
                               255 registers a thread), 1 = the one for two (128) */
    int tn_ctas_per_sm;     /* split-K target of the weighted TN products: CTAs per SM, 1..8 */
    int density_chunks;     /* band chunks per spin of the density pass */
    int lagrange_solver;    /* more than 32 bands: 1 = 4 x 4 tiled cluster, 2 = column
                               cluster; 0 for the single-CTA solver of <= 32 bands */
} cpsd_gpu_tuning;
int cpsd_gpu_get_tuning(const cpsd_gpu_ctx *c, cpsd_gpu_tuning *t);
/* Largest accepted value of every field (lagrange_solver 1 needs a device that
 * schedules its 16-CTA clusters). */
int cpsd_gpu_tuning_limits(const cpsd_gpu_ctx *c, cpsd_gpu_tuning *max);
/* CPSD_ERR_ARG for a value out of range (nothing is changed then). */
int cpsd_gpu_set_tuning(cpsd_gpu_ctx *c, const cpsd_gpu_tuning *t);

/*
 * The project's autotuner: times `steps` SD steps (best of three, captured
 * graphs) for the candidates of one field at a time on this context's own
 * cell -- both plane builds per pass, density chunk counts around the SM-wave
 * model, split-K targets 1, 2 and 4, the two cluster Lagrange solvers -- and
 * keeps a choice that is at least 2% faster.  The result is cached per
 * process by shape (device, grid, bands, sphere, projectors, precision,
 * product engine, learned step, ion motion): a later context of the same
 * shape takes it without timing unless `force`.  Needs the tables and a
 * state; the orbitals and step counters are restored, so call it after
 * cpsd_gpu_set_state and before cpsd_gpu_run (the other outputs of a run are
 * not kept).  ms_before / ms_after (may be NULL): ms per SD step of the
 * choices on entry and of the ones kept (-1 when taken from the cache).
 */
int cpsd_gpu_autotune(cpsd_gpu_ctx *c, int steps, int force, float *ms_before, float *ms_after);

/* CUDA stream the context runs on (a cudaStream_t), for timing with events. */
void *cpsd_gpu_stream(cpsd_gpu_ctx *c);

void cpsd_gpu_destroy(cpsd_gpu_ctx *c);

/* ------------------------------------------------------ learned preconditioner */

/*
 * A 4 -> 64 -> 64 -> 64 -> 1 tanh network (BF16 weights, FP32 accumulate)
 * that maps, per band and |G| shell, (shell kinetic energy / band kinetic
 * energy, log band kinetic energy, log band residual, step feature) to the
 * log of a scale of the SD step.  Training runs on the GPU (hand-written
 * forward, backward and Adam kernels); inputs are host arrays of n x 4
 * floats, targets n floats.
 */
typedef struct cpsd_mlp cpsd_mlp;
int cpsd_mlp_nparams(void);
int cpsd_mlp_create(unsigned long long seed, cpsd_mlp **out);
int cpsd_mlp_forward(cpsd_mlp *m, const float *X, int n, float *y);
/* mean-squared-error loss and its gradient with respect to the FP32 parameters */
int cpsd_mlp_gradient(cpsd_mlp *m, const float *X, const float *T, int n, float *grad, float *loss);
/* `steps` Adam steps over contiguous minibatches of the (pre-shuffled) data */
int cpsd_mlp_train(cpsd_mlp *m, const float *X, const float *T, int n, int steps, int batch, float lr,
                   float *losses);
int cpsd_mlp_get_params(const cpsd_mlp *m, float *p);
int cpsd_mlp_set_params(cpsd_mlp *m, const float *p);
void cpsd_mlp_destroy(cpsd_mlp *m);

/*
 * Attach a network (or NULL for the reference's plain SD): each step then
 * updates c2 = c1 + dte (cpsi + (K(band, shell) - 1) R) instead of
 * c2 = c1 + dte cpsi, before the Lagrange correction, with
 * R = cpsi - C1 (C1' W cpsi) the residual outside the occupied subspace.
 * Where R = 0 the step is plain SD's, so the fixed point (H psi = psi Lambda)
 * is unchanged; the caller keeps plain SD as the fallback when an energy
 * rises.  No counterpart in the reference (its update is cpsd.c:398-400).
 */
int cpsd_gpu_set_preconditioner(cpsd_gpu_ctx *c, cpsd_mlp *m);
/* Select the TN-product engine of the mixed-precision path (CPSD_GEMM_*).
 * The hml product of the energies stays FP64.  The tensor-core modes need a
 * context created with CPSD_PREC_MIXED and have no effect while it runs
 * FP64. */
int cpsd_gpu_set_gemm(cpsd_gpu_ctx *c, int mode);
/* Range [min_log_k, max_log_k] of the learned log step scale, inside
 * [-2, 4.5] (attaching a network opens it fully).  A caller narrows the upper
 * end as a trust region and sets [0, 0] for plain SD steps (K = 1).  Read on
 * the device at every step, so it takes effect without re-capturing the
 * step graphs. */
int cpsd_gpu_set_preconditioner_range(cpsd_gpu_ctx *c, double min_log_k, double max_log_k);
/*
 * The guarded learned loop with plain SD as the arbiter, in the library (no
 * counterpart in the reference): `blocks` blocks of `inner` steps with the
 * attached network (CPSD_ERR_ARG without one), the bound on log K at most
 * *cap.  A block whose energy rises above the previous one (E[0] in), is not
 * finite, or whose Lagrange iteration did not converge (more than one band
 * per spin) is redone from its start with plain SD steps (K = 1: the
 * reference's update), and *cap shrinks by 0.7; an accepted block grows it by
 * 0.1 (within [-2, 4.5]).  E, deltae, deltac: those of the last block;
 * *rejected (may be NULL) counts the redone blocks.  The rollback point is
 * the device copy of cpsd_gpu_save_orbitals.
 */
int cpsd_gpu_run_guarded(cpsd_gpu_ctx *c, int blocks, int inner, double *cap, double *E, double *deltae,
                         double *deltac, int *rejected);

/* Keep a device copy of the current orbitals and step count / go back to it
 * (the rollback point of a guarded block, without a round trip through the
 * host). */
int cpsd_gpu_save_orbitals(cpsd_gpu_ctx *c);
int cpsd_gpu_restore_orbitals(cpsd_gpu_ctx *c);

/* Packed orbitals (ne0+ne1 bands x npw complex, sphere order) out and in. */
int cpsd_gpu_get_packed(cpsd_gpu_ctx *c, double *c1, double *c2, double *cpsi);
int cpsd_gpu_set_packed(cpsd_gpu_ctx *c, const double *c2);
/* The sphere: half-box index, Gamma-point weight and |G| shell of every point. */
int cpsd_gpu_get_sphere(const cpsd_gpu_ctx *c, int *pt_idx, double *weights, int *shell);

/* ------------------------------------------------------ batches of cells */

typedef struct cpsd_gpu_batch cpsd_gpu_batch;

/*
 * Step many independent cells together (uneven grids and band counts
 * allowed).  Each SD step of the whole batch is one CUDA graph launch with
 * one branch per cell.  The cells keep their own contexts (tables and state
 * set beforehand) and must not be run on their own while batched.
 */
int cpsd_gpu_batch_create(cpsd_gpu_ctx **cells, int ncells, cpsd_gpu_batch **out);

/* `inner` SD steps of every cell, then each cell's energies: E[10*i + k] is
 * E[k] of cell i (E[10*i] in: the cell's previous total energy). */
int cpsd_gpu_batch_run(cpsd_gpu_batch *b, int inner, double *E, double *deltae, double *deltac);

/* out[0]: kernel launches of the batch's cells so far. */
void cpsd_gpu_batch_counters(const cpsd_gpu_batch *b, long long *out);
void *cpsd_gpu_batch_stream(cpsd_gpu_batch *b);
void cpsd_gpu_batch_destroy(cpsd_gpu_batch *b);

/*
 * Weighted Gamma-point overlaps as one matrix product, on device memory:
 *   C[i*ldc + j] = sum_{k<K} w[k/2] A[i*lda + k] B[j*ldb + k]   (i < M, j < N)
 * with K reals per row (interleaved re/im of packed coefficients) and one
 * weight per complex pair (w = NULL: all ones).  Each entry is the gcdotc()
 * of ccpsdv3/gcdotc.c:15-28 between rows i and j; ccpsdv3/cpsd.c:420-431
 * builds s22, s21, s12 and s11 from such products, one pair at a time.
 * method: CPSD_GEMM_FP64 or CPSD_GEMM_TF32X3.  Runs on `stream` (NULL: the
 * legacy stream) of the current device and returns after it finishes; the
 * split-K workspace is allocated and freed inside the call.
 */
int cpsd_overlap_tn(int method, int M, int N, int K, const double *A, long lda, const double *B, long ldb,
                    const double *w, double *C, long ldc, void *stream);

/* Largest M*N that cpsd_overlap_tn_noalloc accepts (its split-K workspace,
 * in doubles: 8 MiB less a 256-byte status word). */
#define CPSD_NOALLOC_MAX_DOUBLES 1048544

/*
 * cpsd_overlap_tn without any device allocation.  No counterpart in the
 * reference: an addition for callers that cannot allocate device memory at
 * this point, such as a host code that hands all of the GPU's memory to its
 * own pool at start-up (plane-wave codes sized to the 180 GB of a B200 do),
 * or a caller that must not let cudaMalloc/cudaFree synchronise the device
 * while its other streams are working.
 *
 * Same arguments, method and result as cpsd_overlap_tn (device pointers;
 * returns after `stream` finishes).  The split-K workspace is a file-scope
 * device array of CPSD_NOALLOC_MAX_DOUBLES doubles plus a 256-byte status
 * word, 8 MiB that every GPU which loads this library holds until the
 * process exits; the call makes no cudaMalloc, cudaFree or other allocating
 * call.  Limit: M*N <= CPSD_NOALLOC_MAX_DOUBLES, else CPSD_ERR_SCRATCH and
 * nothing is launched.
 *
 * The first call on each device does a set-up: with that device current it
 * looks up the array's device address (cudaGetSymbolAddress) and sets the
 * tensor-core kernel's shared-memory limit.  A caller that captures streams
 * into CUDA graphs should make that first call before any capture begins.
 * The set-up is kept for the life of the process: a host program that calls
 * cudaDeviceReset (or otherwise destroys the device's primary context) must
 * not call this entry point on that device afterwards, since the cached
 * address belonged to the destroyed context.
 * Every call on a device shares the one array, which keeps the last call's
 * contents: each call clears the status word, and every partial is written
 * before it is read.  Calls whose GPU work overlaps (on concurrent streams,
 * or from several host threads) race on the array: serialise them.
 */
int cpsd_overlap_tn_noalloc(int method, int M, int N, int K, const double *A, long lda, const double *B,
                            long ldb, const double *w, double *C, long ldc, void *stream);

#ifdef __cplusplus
}
#endif
#endif
