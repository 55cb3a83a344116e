/*
 * green-b200: B200-native (sm_100a) HF-exchange and GW self-energy kernels.
 *
 * C ABI of libgreen_b200.so.  Plain pointers and sizes only; every function
 * returns an int status (GG_OK = 0) and never lets a C++ exception cross the
 * boundary.  Complex numbers are interleaved (re, im) double pairs, i.e. the
 * memory layout of std::complex<double>; all tensors are row-major (C order),
 * the layout the reference's ndarray/Eigen::RowMajor tensors use.
 *
 * Which reference interface each entry point replaces (paths relative to the
 * Green-Phys/green-gpu tree):
 *
 *   gg_create / gg_destroy        kernel object lifetime behind the shared_ptr<void>
 *                                 returned by custom_gw_kernel / custom_hf_kernel
 *                                 (src/green/gpu/gpu_factory.h:47-89) and the device
 *                                 set-up of cugw_utils / cuhf_utils
 *                                 (src/cugw_utils.cu:27-75, src/cuhf_utils.cu:31-72)
 *   gg_set_symmetry               cu_symmetry::initialize (src/cu_symmetry.cu:36-140) fed
 *                                 by make_cu_symmetry_data (src/gw_gpu_kernel.cpp:34-91)
 *   gg_set_kpairs, gg_set_coulomb the integral store df_integral_t::read_entire /
 *   gg_set_coulomb_device         symmetrize (src/green/gpu/df_integral_t.h:96-235)
 *   gg_set_ir                     allocate_IR_transformation_matrices
 *                                 (src/cuda_common.cu:93-108; Ttn_FB / Tnt_BF of
 *                                 grids::transformer_t used at src/cugw_utils.cu:35)
 *   gg_gw_sigma                   gw_gpu_kernel::solve (src/gw_gpu_kernel.cpp:163-205),
 *                                 i.e. the callback of custom_gw_kernel
 *                                 (src/green/gpu/gpu_factory.h:86-87)
 *   gg_hf_exchange                cuhf_utils::accumulate_exchange_on_device
 *                                 (src/cuhf_utils.cu:136-159)
 *   gg_hf_fock                    hf_gpu_kernel::solve (src/hf_gpu_kernel.cpp:66-104),
 *                                 i.e. the callback of custom_hf_kernel
 *                                 (src/green/gpu/gpu_factory.h:50-61)
 *   gg_symmetry_unfold            cu_symmetry::transform_k_ao_device
 *                                 (src/cu_symmetry.cu:183-233)
 */
#ifndef GREEN_B200_H
#define GREEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define GG_OK 0
#define GG_ERR_ARG 1       /* invalid argument or shape mismatch */
#define GG_ERR_CUDA 2      /* CUDA runtime error (message has the call and file:line) */
#define GG_ERR_NOT_HPD 3   /* Cholesky: I - P~ is not Hermitian positive definite */
#define GG_ERR_SINGULAR 4  /* LU: exactly singular I - P~ */
#define GG_ERR_STATE 5     /* a required input (symmetry, integrals, IR) was not set */
#define GG_ERR_MEMORY 6    /* the system does not fit the device memory budget */
#define GG_ERR_INTERNAL 7

/* linear solver for (I - P~) W~ = P~ (LinearSolverType, src/green/gpu/common_defs.h:137-139) */
#define GG_SOLVER_CHOLESKY 0
#define GG_SOLVER_LU 1

/* arithmetic of the contractions */
#define GG_PREC_FP64 0     /* plain FP64 everywhere */
#define GG_PREC_SPLIT 1    /* Ozaki-sliced INT8 tensor-core contractions, FP64 solve / IR / sums */
#define GG_DEFAULT_SPLIT_SLICES 5

typedef struct gg_context gg_context;

typedef struct gg_shape {
  int32_t nk;    /* full-BZ k points */
  int32_t ink;   /* irreducible k points */
  int32_t nq;    /* full-BZ q points (== nk) */
  int32_t inq;   /* irreducible q points */
  int32_t nao;   /* orbitals per spin block */
  int32_t NQ;    /* auxiliary (density-fitting) basis size */
  int32_t ns;    /* spins (1 or 2) */
  int32_t nts;   /* imaginary-time points incl. 0 and beta; even */
  int32_t nw_b;  /* bosonic Matsubara frequencies; nw_b <= nts */
  int32_t reserved;
} gg_shape;

/* Create a context on CUDA device `device`.  Allocates no per-iteration state yet. */
int gg_create(const gg_shape* shape, int device, gg_context** out);
void gg_destroy(gg_context* ctx);
/* Message of the last failing call on this context (or, when ctx is NULL, of the last
 * failing context-free call on this thread: gg_create or gg_zgemm_noalloc).  Valid until
 * the next call on the same context / thread. */
const char* gg_last_error(const gg_context* ctx);

/* Symmetry tables (cu_symmetry_data, src/green/gpu/cu_symmetry.h:41-66).  All index
 * arrays are int64.  k1_from_k2q / k2_from_k1q are flattened [k * nq + q].  U_k is
 * complex [nk][nao][nao], U_q complex [nq][NQ][NQ]; pass NULL for identity rotations.
 * Stars are the full-BZ points with the same reduced index, in ascending order. */
int gg_set_symmetry(gg_context* ctx, const int64_t* k_full_to_reduced, const int64_t* k_reduced_to_full,
                    const int64_t* k_tr_conj, const int64_t* q_full_to_reduced,
                    const int64_t* q_reduced_to_full, const int64_t* q_tr_conj, const int64_t* k1_from_k2q,
                    const int64_t* k2_from_k1q, const double* U_k, const double* U_q);

/* k-pair store layout (df_integral_t.h:68-86, 153-173): for the triangular index
 * idx = tri(k1 >= k2), conj_kpair_list[idx] / trans_kpair_list[idx] name the stored pair it
 * is the conjugate / transpose of (== idx when none), irre_pos_kpair[idx] is the position
 * of a stored pair in the V array (-1 otherwise).  Arrays have nk(nk+1)/2 entries. */
int gg_set_kpairs(gg_context* ctx, int64_t num_kpair_stored, const int64_t* conj_kpair_list,
                  const int64_t* trans_kpair_list, const int64_t* irre_pos_kpair);

/* Density-fitted integrals V [num_kpair_stored][NQ][nao][nao] complex.  The host variant
 * copies them into device memory owned by the context; the device variant borrows a
 * device pointer that must stay valid for the context's lifetime. */
int gg_set_coulomb(gg_context* ctx, const double* V_stored);
int gg_set_coulomb_device(gg_context* ctx, const void* V_stored_device);

/* IR transforms: Ttn_FB complex [nts][nw_b], Tnt_BF complex [nw_b][nts-2]. */
int gg_set_ir(gg_context* ctx, const double* Ttn_FB, const double* Tnt_BF);

/* Restrict the next GW builds to the irreducible q points iq with iq % size == rank (the
 * round-robin distribution of src/cugw_utils.cu:115); the caller sums the partial Sigma
 * over ranks (src/gw_gpu_kernel.cpp:187).  (0, 1) restores the full build. */
int gg_set_q_shard(gg_context* ctx, int rank, int size);
/* The irreducible q points a shard owns (ascending), as gg_set_q_shard restricts a build to
 * them: writes at most `capacity` indices to q_out and their number to count.  Host-only (no
 * device, no context), so multi-rank drivers can plan the distribution before any GPU work. */
int gg_q_shard_points(int32_t inq, int rank, int size, int32_t* q_out, int32_t capacity, int32_t* count);

/* Number of Ozaki slices per operand for GG_PREC_SPLIT (2..8, default GG_DEFAULT_SPLIT_SLICES).
 * Five slices is the smallest count that keeps Sigma, P0, the exchange K and the energies
 * within 1e-8 relative of the FP64 path on the benchmark systems (four slices gives about
 * 5e-8). */
int gg_set_split_slices(gg_context* ctx, int slices);

/* Form of the last two steps of the Sigma contraction, Z = X G and the reduction of Z V^+
 * over (Q, orbital): enable = 1 runs them as one FP64 tensor-core kernel that keeps Z in
 * registers, for nao <= 52 (larger orbital counts use the two GEMMs); enable = 0 (default) runs
 * the two GEMMs, with Z in device memory, as src/cugw_qkpt.cu:295-332 does.  The fused form
 * saves Z's write and read (2 x nts x NQ x nao^2 x 16 bytes per (k, q) pair), but both forms
 * are bound by the DMMA issue rate, and at nao 52, NQ 400 the fused kernel takes 2.64 ms per
 * pair against 2.54 ms for the two GEMMs.  Both sum in a fixed order (deterministic); they
 * differ in the FP64 summation order only. */
int gg_set_fused_tail(gg_context* ctx, int enable);

/* One GW self-energy build.  G_tskij complex [nts][ns][ink][nao][nao] (host), Sigma_tskij
 * the same shape (host, overwritten: zeroed, accumulated, divided by nk as
 * gw_gpu_kernel::solve does).  solver: GG_SOLVER_*; precision: GG_PREC_*. */
int gg_gw_sigma(gg_context* ctx, const double* G_tskij, double* Sigma_tskij, int solver, int precision);
/* Same with device buffers on the given cudaStream_t (NULL: the context's stream). */
int gg_gw_sigma_device(gg_context* ctx, const void* G_tskij_device, void* Sigma_tskij_device, int solver,
                       int precision, void* stream);

/* Optional capture of intermediates of the next gg_gw_sigma* call (host pointers, any may
 * be NULL): P0 [inq][nts][NQ][NQ] (scaled by 1/nk and mirrored), Pw [inq][nw_b][NQ][NQ]
 * (Hermitian-symmetrised P~), Wt [inq][nts][NQ][NQ] (W~(tau)). */
int gg_set_capture(gg_context* ctx, double* P0_out, double* Pw_out, double* Wt_out);

/* Arithmetic of the HF exchange contraction for the next gg_hf_exchange / gg_hf_fock calls
 * (GG_PREC_FP64 default, GG_PREC_SPLIT: Ozaki INT8 with the context's slice count).  The
 * reference's HF path is FP64 only (cuhf_utils.cu). */
int gg_set_hf_precision(gg_context* ctx, int precision);

/* Two-component (X2C) mode, replacing x2c_gw_gpu_kernel / x2c_hf_gpu_kernel
 * (src/gw_gpu_kernel.cpp:457-551, src/hf_gpu_kernel.cpp:229-338; selected by the X2C flag of
 * custom_gw_kernel / custom_hf_kernel, gpu_factory.h:47-89).  The context is created with
 * ns = 1 and nao = the number of orbitals per spin; G, Sigma, dm, S_k and the Fock matrix are
 * then spinor matrices of order nso = 2 nao: G/Sigma [nts][1][ink][nso][nso], dm/S_k/F
 * [1][ink][nso][nso].  GW runs on the spin blocks aa, bb, ab, ba as four pseudo-spins (P0
 * prefactor -1, the ab block of G(tau) paired with the ba block of G(-tau)); HF on aa, bb, ab
 * (prefactor -1, ba = ab^+), the Hartree term from aa + bb added to aa and bb, Ewald per block
 * with S_aa.  Only the identity k/q symmetry is accepted (GG_ERR_ARG otherwise). */
int gg_set_x2c(gg_context* ctx, int enable);

/* Graph mode for gg_gw_sigma / gg_gw_sigma_device (no counterpart in the reference, which
 * launches every contraction from the host: cugw_utils.cu:104-202).  With graph mode on, the
 * first build runs eagerly and is then captured into one CUDA graph; later builds with the same
 * buffers, stream, solver and precision replay it (one launch instead of tens of thousands).
 * Dyson failures and split-engine time-outs are still reported, after the replay.  Every setter
 * of the context drops the graph; profiling and intermediate capture fall back to eager builds. */
int gg_set_graph(gg_context* ctx, int enable);

/* Several systems (contexts of any shape on one device) built in one CUDA graph: each system's
 * build runs on its own context stream, so their kernels overlap on the device.
 * gg_batch_create runs every build once eagerly (the results are valid) and captures them;
 * gg_batch_run replays all of them (stream NULL: the batch's own stream) and returns the first
 * failure (message through gg_last_error(NULL)).  G[i] / Sigma[i] are device buffers of system i
 * in its layout; the contexts must not be changed while the batch exists. */
typedef struct gg_batch gg_batch;
int gg_batch_create(gg_context* const* ctxs, int n, const void* const* G_device, void* const* Sigma_device,
                    int solver, int precision, gg_batch** out);
int gg_batch_run(gg_batch* batch, void* stream);
void gg_batch_destroy(gg_batch* batch);

/* Exchange part K_s(k) [ns][ink][nao][nao] for the IBZ density dm [ns][ink][nao][nao]
 * (host buffers). */
int gg_hf_exchange(gg_context* ctx, const double* dm, double* K_out);
/* Full static self-energy of hf_gpu_kernel::solve: exchange (GPU) + direct + Ewald
 * (S_k [ns][ink][nao][nao]).  Host buffers. */
int gg_hf_fock(gg_context* ctx, const double* dm, const double* S_k, double madelung, double* F_out);

/* X(k) = U_k X(k_ibz) U_k^+ (conjugated for time-reversal partners) for every full-BZ k:
 * X_ibz [nmat][ink][nao][nao] -> X_full [nmat][nk][nao][nao]; host buffers. */
int gg_symmetry_unfold(gg_context* ctx, const double* X_ibz, int64_t nmat, double* X_full);

/* Seconds spent in each phase of the last GW build (device time, CUDA events):
 * out[0] total, [1] G unfold, [2] P0, [3] IR forward, [4] Dyson, [5] IR back, [6] Sigma,
 * [7] end to end of the last host-buffer call (gg_gw_sigma: H2D copy of G, build, D2H of
 * Sigma).
 * Returns the number of entries written (<= n). */
int gg_last_timings(const gg_context* ctx, double* out, int n);

/* Per-kernel device time of the last GW build, from CUDA events recorded around every
 * launch of the named contraction on its stream when profiling is enabled:
 * which = 0: the P0 contraction (sum over k of A_k B_k^T), 1: the Sigma contraction
 * (V times W~), 2: the final Sigma product with V^+ (reduction over Q and an orbital), or with
 * gg_set_fused_tail the fused kernel that also forms its operand Z = X G.  Each entry covers
 * launches of one kernel kind.
 * Writes launches, total seconds and algorithmic flops
 * (8MNK + 12MN per complex GEMM, src/green/gpu/common_defs.h:121-125). */
int gg_set_profiling(gg_context* ctx, int enable);
int gg_kernel_stats(const gg_context* ctx, int which, int64_t* launches, double* seconds, double* flops);
/* Number of kernel launches issued by the last GW build or HF call. */
int64_t gg_last_launch_count(const gg_context* ctx);

/* Dense complex GEMM with the library's engines: C = A B for row-major A [M][K],
 * B [K][N], C [M][N] (host buffers).  precision GG_PREC_FP64 runs the FP64 tensor-core
 * engine, GG_PREC_SPLIT the Ozaki INT8 engine with the context's slice count.  Same
 * arithmetic as the contractions inside gg_gw_sigma / gg_hf_exchange (no reference
 * counterpart: it exposes the engine for accuracy studies). */
int gg_zgemm(gg_context* ctx, int64_t M, int64_t N, int64_t K, const double* A, const double* B, double* C,
             int precision);

/* C = A B for device buffers A [M][K], B [K][N], C [M][N] (row-major complex128, 16-byte
 * aligned), FP64 tensor-core engine, enqueued on `stream` (a cudaStream_t; NULL = legacy
 * default stream) without synchronising.  No counterpart in the reference: this entry
 * point exists for callers that may not allocate device memory where they call it -
 * programs whose device memory belongs to another allocator or to a budget fixed at
 * start-up, and latency-bound loops in which cudaMalloc's implicit device synchronisation
 * would stall other streams.  It allocates nothing: the
 * split-K partial sums live in a static 16 MiB device array (2^20 complex numbers) that
 * every GPU loading this library keeps until the process exits, so M * N may not exceed
 * 2^19 (larger sizes return GG_ERR_ARG with the limit in gg_last_error(NULL)).  The first
 * call on each device looks the array's address up once (cudaGetSymbolAddress with that
 * device current); make that first call before any stream capture, and do not call it again
 * on a device after a cudaDeviceReset in the same process.  All calls share the
 * array and every value a call reads from it was written earlier in the same call, so
 * nothing needs clearing - but calls that overlap on the GPU (different streams, or
 * different host threads on one device) race on it and must be serialised by the caller. */
int gg_zgemm_noalloc(int64_t M, int64_t N, int64_t K, const void* A, const void* B, void* C, void* stream);

/* FP64 energy and chemical-potential reductions.  green-gpu returns Sigma(tau) and the Fock
 * matrix and leaves these reductions to its caller, green-mbpt (its GW / HF solvers read
 * the kernels' outputs and reduce them in double precision); they are provided here so that a
 * caller of this library keeps them in FP64 next to the data.  k weights are |star(k)| / nk
 * from the context's symmetry tables; the spin factor f is 2 for ns = 1, 1 for ns = 2 and in
 * X2C mode (where the matrices are the spinor ones).
 *   gg_energy_hf: dm, H (one-body Hamiltonian) and F (Fock matrix) [ns][ink][m][m] host;
 *     out[0] = E_1b = f sum_{s,k} w_k Re Tr(dm H), out[1] = E_HF = (f/2) sum w_k Re Tr(dm (H + F)).
 *   gg_energy_gw[_device]: G and Sigma [nts][ns][ink][m][m] (host, or device buffers on
 *     `stream`), M [nts][nts] real (host) a bilinear quadrature of
 *     int_0^beta f(tau) g(beta - tau) dtau on the tau grid; *e_gw = -(f/2) sum_{s,k} w_k
 *     sum_{t,t'} M[t][t'] Re Tr(Sigma(tau_t) G(tau_t')) (Galitskii-Migdal), traces on the FP64
 *     tensor-core engine. */
int gg_energy_hf(gg_context* ctx, const double* dm, const double* H, const double* F, double* out);
int gg_energy_gw(gg_context* ctx, const double* G_tskij, const double* Sigma_tskij, const double* M,
                 double* e_gw);
int gg_energy_gw_device(gg_context* ctx, const void* G_tskij_device, const void* Sigma_tskij_device,
                        const double* M, double* e_gw, void* stream);
/* Chemical potential of a mean-field state: the mu with
 * spin_factor sum_{s,k} weights[k] sum_n 1 / (1 + exp(beta (e_skn - mu))) = nelec, where e_skn
 * are the eigenvalues of F_s(k) x = e S_s(k) x (F, S complex [ns][ink][n][n], host), found by a
 * Cholesky reduction and cyclic Jacobi in FP64 and bisected to FP64 resolution.  *n_at_mu (may
 * be NULL) receives the particle number at the result.  Host-only, context-free. */
int gg_chemical_potential(int32_t ns, int32_t ink, int32_t n, const double* weights, const double* F,
                          const double* S, double beta, double spin_factor, double nelec, double* mu,
                          double* n_at_mu);

/* Device bytes a context of this shape needs when its integrals are resident and its GW
 * work space is planned without chunking (V store of num_kpair_stored pairs + work space);
 * context-free, allocates nothing.  Used for admission by memory footprint. */
int gg_estimate_bytes(const gg_shape* shape, int64_t num_kpair_stored, int64_t* bytes);

/* Tile autotuner of the split-precision INT8 engine (no counterpart in the reference, whose
 * GEMMs are cuBLAS calls).  With it enabled, the first call of every distinct GEMM shape on this
 * context that overwrites its output (beta = 0) and is not being captured into a CUDA graph is
 * run for every candidate tile width (96 / 80 / 64 / 48 B' rows at 5 slices) and split-K factor
 * (the wave-filling rule's, one, twice the rule's) - once untimed, once timed with CUDA events on
 * the call's stream;
 * that call's result and every later call of the shape use the fastest.  Tile width does not
 * change any element's arithmetic; split-K changes only the FP64 summation order of the partial
 * sums.  gg_autotune_report returns one line per tuned shape (valid until the next call on the
 * context).  Disabling clears the choices. */
int gg_set_autotune(gg_context* ctx, int enable);
const char* gg_autotune_report(const gg_context* ctx);

/* Test hook of the split engine's time-out path (no counterpart in the reference, whose device
 * lock spins without a limit: src/cuda_common.cu:225-231).  The next split-precision GEMM on
 * this context runs with a 0.1 s limit on every barrier wait, and one epilogue warp of CTA 0
 * withholds its release of the first accumulator it drains, so the MMA warp's wait for that
 * accumulator runs out (the GEMM needs more work units than SMs).  The kernel records the
 * time-out, waits (bounded) for its copies and MMAs in flight, frees its tensor memory and
 * returns; the call reports GG_ERR_INTERNAL and the context stays usable.  One-shot. */
int gg_arm_split_timeout_test(gg_context* ctx);

/* Library build information string (static storage). */
const char* gg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GREEN_B200_H */
