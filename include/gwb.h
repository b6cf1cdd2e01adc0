/*
 * gwb.h - C ABI of the B200 (sm_100a) Kohn-Sham band-solve library libgwb.so.
 *
 * The library replaces the hot path of gradwave's plane-wave band solve: the
 * batched Hamiltonian apply H psi and the block-Davidson steps around it.
 * Every entry point:
 *   - takes plain pointers and sizes (no torch types); array arguments are
 *     DEVICE pointers unless the comment says host;
 *   - is stream ordered on the cudaStream_t passed as `void* stream`
 *     (NULL = legacy default stream) and does not synchronise the host unless
 *     the comment says so;
 *   - returns an int status (GWB_OK = 0); gwb_last_error() gives the message
 *     of the last failure on the calling thread. No C++ exception crosses it.
 *
 * Layouts (row-major, the reference's, gradwave core/batch.py:1-14):
 *   coefficient blocks c       (nk, nb, npw_max) complex, padded slots 0
 *   kinetic t                  (nk, npw_max) float64, 0 in padding
 *   flat_idx                   (nk, npw_max) int64 box index
 *                              i0*n1*n2 + i1*n2 + i2 (gradwave grids.py:171)
 *   v_eff_r                    (n0, n1, n2) float64 [eV]
 *   projectors p               (nk, nproj, npw_max) complex128, 0 in padding
 *   dij                        (nproj, nproj) float64 [eV]
 * Complex numbers are interleaved (re, im) pairs of float64 (GWB_C128) or
 * float32 (GWB_C64), i.e. torch.complex128 / torch.complex64 storage.
 *
 * Handles are thread-compatible: one handle per host thread at a time.
 */
#ifndef GWB_H_
#define GWB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GWB_OK 0
#define GWB_ERR_ARG 1          /* bad shape, size or pointer */
#define GWB_ERR_CUDA 2         /* a CUDA runtime or library call failed */
#define GWB_ERR_NONFINITE 3    /* NaN/Inf found where a finite value is required */
#define GWB_ERR_TIMEOUT 4      /* a bounded device wait ran out */
#define GWB_ERR_NOT_CONVERGED 5
#define GWB_ERR_ALLOC 6        /* device allocation failed */
#define GWB_ERR_BREAKDOWN 7    /* Cholesky of a non positive-definite Gram matrix */

/* io dtypes */
#define GWB_C64 0
#define GWB_C128 1
/* compute precisions */
#define GWB_FP32 0
#define GWB_FP64 1

/* Message of the last failure on this thread ("" if none). */
const char* gwb_last_error(void);
/* Library version string. */
const char* gwb_version(void);
/* Number of kernels this library has launched in the process so far. */
unsigned long long gwb_launch_count(void);

/* ======================================================================= */
/* Hamiltonian apply                                                       */
/* ======================================================================= */

typedef struct gwb_ham gwb_ham;

/* Geometry of one k batch (HOST arrays, copied at create). */
typedef struct {
  int32_t nk;
  int32_t npw_max;
  int32_t n[3];            /* FFT box n0, n1, n2: each 2^a 3^b 5^c 7^d, <= 128 */
  int32_t nproj;           /* Kleinman-Bylander projector columns (may be 0) */
  const int64_t* npw;      /* (nk) true plane-wave count per k */
  const int64_t* flat_idx; /* (nk*npw_max) box index of every sphere point */
} gwb_ham_geometry;

/* Replaces: gradwave core/batch.py:249-304 (BatchedHamiltonian.__init__: the
 * persistent scatter box with its trash slot and the cached tables). Builds the
 * sphere -> box-plane maps and allocates handle-owned scratch on `device`. */
int gwb_ham_create(const gwb_ham_geometry* geom, int device, gwb_ham** out);
int gwb_ham_destroy(gwb_ham* h);

/* Kinetic diagonal t (nk*npw_max float64, device). Replaces the t table of
 * gradwave core/batch.py:306-331 (_tables). */
int gwb_ham_set_kinetic(gwb_ham* h, const double* t, void* stream);
/* Local potential v(r) (n0*n1*n2 float64, device). Replaces v_eff of
 * gradwave core/batch.py:306-331. */
int gwb_ham_set_potential(gwb_ham* h, const double* v_eff_r, void* stream);
/* Projectors (complex128, device) and D (float64, device). Replaces p, p_conj
 * and dij of gradwave core/batch.py:306-331. */
int gwb_ham_set_projectors(gwb_ham* h, const void* p, const double* dij, void* stream);

/* out = H c over all k and nb bands, padded slots of out set to 0.
 * Replaces gradwave core/batch.py:480-505 (BatchedHamiltonian.apply).
 *   io_dtype: storage of c and out (GWB_C64 / GWB_C128)
 *   prec:     arithmetic of the FFTs, kinetic and nonlocal terms
 *             (GWB_FP32 / GWB_FP64); GWB_FP64 with GWB_C64 storage is allowed.
 * c and out must not overlap. */
int gwb_ham_apply(gwb_ham* h, const void* c, void* out, int32_t nb, int32_t io_dtype,
                  int32_t prec, void* stream);

/* As gwb_ham_apply with explicit distances (in complex elements) between the
 * k blocks of c and of out, so a band slice of a larger (nk, m, npw_max) block
 * (the Davidson basis) can be read or written in place. Each k block holds nb
 * contiguous rows of npw_max. */
int gwb_ham_apply_strided(gwb_ham* h, const void* c, int64_t c_kstride, void* out, int64_t out_kstride,
                          int32_t nb, int32_t io_dtype, int32_t prec, void* stream);

/* Tuning of a handle's applies (0 keeps the built-in rule): the bytes of FFT
 * scratch per band chunk (default 48 MiB or GWB_W_BUDGET_MB: chunks of bands
 * whose scratch stays in L2) and the number of CTAs the G-sliced projector
 * contraction aims for (default 4 x 148). The values are chosen per box and
 * projector count by gradwave_b200.autotune from timed applies. No
 * counterpart in the reference. */
int gwb_ham_set_tuning(gwb_ham* h, int64_t w_budget_bytes, int32_t nl_target_ctas);
/* Threads per block of the shared-memory FFT kernels of the 72^3 and 96^3
 * boxes, per arithmetic precision: 256, 512 or 1024 (0: the built-in 512 for
 * float32, 1024 for float64). One block of a float64 96^3 plane fills the
 * shared memory of an SM, so more threads per block means more warps to hide
 * the latency of its barrier-separated passes. */
int gwb_ham_set_fft_threads(gwb_ham* h, int32_t threads_fp32, int32_t threads_fp64);

/* Augmentation matrix q (nproj*nproj float64, real symmetric, device) of the
 * overlap S = 1 + sum_pq |beta_p> q_pq <beta_q| (USPP/PAW). Set after the
 * projectors. Replaces q_full of gradwave scf/uspp_batch.py:34-45
 * (BatchedHS.__init__). */
int gwb_ham_set_overlap(gwb_ham* h, const double* q, void* stream);

/* out_h = H c and out_s = S c in one pass (the projector contraction
 * <beta|c> is formed once and feeds both the D and the q terms; padded slots
 * of both outputs are 0). Strides as in gwb_ham_apply_strided; c, out_h and
 * out_s must not overlap. Replaces gradwave scf/uspp_batch.py:56-73
 * (BatchedHS.h and BatchedHS.s applied to the same block). */
int gwb_ham_apply_hs(gwb_ham* h, const void* c, int64_t c_kstride, void* out_h, int64_t oh_kstride, void* out_s,
                     int64_t os_kstride, int32_t nb, int32_t io_dtype, int32_t prec, void* stream);

/* Electron density on the box: rho[r] = scale * sum_k sum_b weights[k*w_kstride + b]
 * |psi_kb(r)|^2 with psi_kb(r) = sum_G c_kb(G) exp(iG.r) (the unnormalised
 * inverse FFT of the sphere coefficients; padded slots of c must be zero, as
 * they are in the eigenvectors). rho is (n0*n1*n2) float64, device; the FFTs
 * and sums run in float64 whatever the storage of c. For gradwave's
 * density_b pass weights = kweights[k] * occ[k, b] and scale = 1 / volume.
 * Needs only the geometry of the handle (no kinetic, potential or
 * projectors), and uses the handle's scratch: do not overlap it with an
 * apply on the same handle. Replaces gradwave core/batch.py:562-587
 * (density_b) with g_to_r_b (core/batch.py:208-216). */
int gwb_ham_density(gwb_ham* h, const void* c, int64_t c_kstride, int32_t nb, int32_t io_dtype,
                    const double* weights, int64_t w_kstride, double scale, double* rho, void* stream);

/* Gamma point in the real embedding of the half sphere (replaces gradwave
 * core/gamma.py:161-250, GammaHamiltonian.apply composed with embed_real and
 * unembed_real). The handle is a k = 0 operator on the full sphere (nk = 1,
 * npw_max = npw = 2 nhalf - 1, no padding). phi and out are nb rows of
 * 2 nhalf - 1 float64 (row strides ldphi, ldout): phi = (Re c(0),
 * sqrt2 Re c(G1), sqrt2 Im c(G1), ...) over the representatives G0 = 0, G1, ...
 * Index tables (device int32 / uint8, from the reference's half-sphere maps):
 *   src_half[g]    half slot of full-sphere point g (its representative)
 *   conj_full[g]   1 where c(g) is the conjugate of its representative
 *   rep_full[j]    full-sphere index of representative j
 *   partner_rep[j] full-sphere index of -G_j (j = 0: itself)
 * Two real bands run as one complex row of the apply (z = c_a + i c_b),
 * unpacked by the G / -G symmetry: half the FFT and nonlocal work per band.
 * prec: GWB_FP64 or GWB_FP32 arithmetic of the apply. work: at least
 * gwb_gamma_work_bytes(nb, npw) bytes of device memory. */
size_t gwb_gamma_work_bytes(int32_t nb, int32_t npw);
int gwb_gamma_apply(gwb_ham* h, int32_t nb, int32_t nhalf, int32_t npw, const double* phi, int64_t ldphi,
                    double* out, int64_t ldout, const int32_t* src_half, const uint8_t* conj_full,
                    const int32_t* rep_full, const int32_t* partner_rep, int32_t prec, void* work,
                    size_t work_bytes, void* stream);

/* Bytes of handle-owned device scratch currently held. */
size_t gwb_ham_scratch_bytes(const gwb_ham* h);

/* Float32 applies of complex128 blocks with nproj >= 128 run the nonlocal
 * term as split-BF16 tensor-core products (gwb_zgemm_tc; error ~1e-6 of the
 * term, below the float32 arithmetic of the rest; GWB_TC_NONLOCAL=0 in the
 * environment keeps the CUDA-core kernels). This reads (synchronously) and
 * clears the handle's record of a timed-out pipeline wait in them: *status
 * = 0 and GWB_OK if none, else GWB_ERR_TIMEOUT. */
int gwb_ham_tc_status(gwb_ham* h, int* status);

/* ======================================================================= */
/* Davidson steps (complex128 blocks, float64 reductions)                  */
/* A "k stride" is the distance in complex elements between the blocks of   */
/* consecutive k; rows inside a block are npw apart.                        */
/* ======================================================================= */

/* Batched row-major complex128 GEMM: C = alpha op(A) op(B) + beta C per batch,
 * op 0 = N, 1 = T, 2 = H; op(A) is M x K, op(B) K x N. Plain cuBLAS ZGEMM.
 * Replaces the torch.matmul/einsum products of gradwave
 * solvers/davidson.py:428-432,648-654,752-756. */
int gwb_zgemm(int opA, int opB, int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im,
              const void* A, int64_t lda, int64_t strideA, const void* B, int64_t ldb, int64_t strideB,
              double beta_re, double beta_im, void* C, int64_t ldc, int64_t strideC, int64_t batch,
              void* stream);

/* C = alpha A B^H + beta C per batch for row-major A (M x K), B (N x K) with
 * a long reduction K (plane waves) and a small output: K is split into slices
 * accumulated in `work` (at least M*N*batch*16 bytes; more bytes allow more
 * slices), then summed in a fixed order. The subspace, projection and Gram
 * products of gradwave solvers/davidson.py:428-432,648-649,215. */
int gwb_zgemm_nh(int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im, const void* A, int64_t lda,
                 int64_t strideA, const void* B, int64_t ldb, int64_t strideB, double beta_re, double beta_im,
                 void* C, int64_t ldc, int64_t strideC, int64_t batch, void* work, size_t work_bytes,
                 void* stream);

/* Split-precision complex products on the tensor cores (tcgen05, BF16
 * operands, FP32 accumulation in tensor memory). An operand is a "plane set":
 * per batch entry four BF16 planes re_hi, re_lo, im_hi, im_lo (x = hi + lo to
 * about 2^-17 |x|), each rows_cap x ld (ld a multiple of 8, 16-byte aligned
 * base), plane q of entry b at element (4 b + q) * rows_cap * ld.
 *
 * gwb_tc_planes: rows [0, rows) x cols of complex src (dtype GWB_C64 or
 * GWB_C128, row stride src_ld, batch stride src_kstride, elements; conj != 0
 * stores the conjugate) into plane rows [row0, row0 + rows), columns cols..ld-1
 * zeroed. */
int gwb_tc_planes(int64_t nk, int64_t rows, int64_t cols, const void* src, int64_t src_ld, int64_t src_kstride,
                  int dtype, int conj, void* planes, int64_t ld, int64_t rows_cap, int64_t row0, void* stream);

/* C = alpha A op(B) + beta C per batch entry (float64 complex C, row-major,
 * ldc / strideC in elements); A: M x K planes; opB = 2: op(B) = B^H with B an
 * N x K plane set; opB = 0: op(B) = B with B a K x N plane set. Twelve BF16
 * tensor-core products per complex multiply-add (re/im x hi/lo), error about
 * 2^-15 sum_k |a_ik||b_kj|. opB = 2 splits K over CTAs when the tile grid is
 * small, with the partial sums in `work` (gwb_zgemm_tc_work_bytes; with less,
 * fewer splits). A wait that runs out ORs GWB_ERR_TIMEOUT into *status (a
 * device int). The products of the first projection pass of the
 * expansion block, gradwave solvers/davidson.py:428-432; no counterpart in
 * the reference's precision choices (it has float64 and float32 only). */
int64_t gwb_zgemm_tc_work_bytes(int opB, int64_t M, int64_t N, int64_t K, int64_t batch);
/* Limit (SM clock cycles, default 4e9, about two seconds) of every mbarrier
 * wait in the tensor-core products, read at each launch; a wait that runs out
 * reports GWB_ERR_TIMEOUT through *status, after the CTA has waited (bounded)
 * for its issued bulk copies and MMAs. No counterpart in the reference. */
int gwb_tc_set_wait_limit(int64_t cycles);
/* Failure-test hook: with kstep >= 0 every later gwb_zgemm_tc launch issues no
 * load for K step kstep of its split, so that step's consumer wait runs out
 * (GWB_ERR_TIMEOUT) without a fault; -1 turns it off. For the tests of the
 * bounded waits only. No counterpart in the reference. */
int gwb_tc_test_withhold(int32_t kstep);
int gwb_zgemm_tc(int opB, int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im, const void* A_planes,
                 int64_t lda, int64_t a_rows_cap, const void* B_planes, int64_t ldb, int64_t b_rows_cap,
                 double beta_re, double beta_im, void* C, int64_t ldc, int64_t strideC, int64_t batch, void* work,
                 size_t work_bytes, int* status, void* stream);

/* Float64-accurate real products on the int8 tensor cores (tcgen05
 * kind::i8, the Ozaki scheme). A slice set is s (6, 7 or 8) int8 planes of
 * rows_cap x ldk (ldk a multiple of 64, 16-byte aligned base), plane p at
 * p rows_cap ldk, with one float64 scale per row: row r is
 * scale[r] sum_p plane_p[r] 2^(-6-7p) to within 2^-7s scale[r], every plane
 * value in [-64, 64] (each rounded to nearest; scale the power of two above
 * the row's largest magnitude). The float64 GEMMs of the Davidson subspace, Ritz, projection
 * and Cholesky-QR steps (gradwave solvers/davidson.py:195-222,428-432,
 * 648-657) run on them; the reference has no counterpart.
 *
 * gwb_oz_split_rows: rows [row0, row0 + rows) of the set from the rows of src
 * (K columns, row stride ld_src), each element times fold[k] when fold is
 * not NULL; columns K..ldk-1 zeroed; scale[row0 + r] set. */
int gwb_oz_split_rows(int32_t s, int64_t rows, int64_t K, const double* src, int64_t ld_src, const double* fold,
                      void* slices, int64_t ldk, int64_t rows_cap, int64_t row0, double* scale, void* stream);
/* gwb_oz_split_cols: the transposed layout. src is krows x R (row stride
 * ld_src); row r of the set gets, in columns k0 .. k0 + krows - 1, the
 * slices of src[k][r] / kscale[k0 + k], with kscale[k0 + k] the power of two
 * above max_r |src[k][r]| (set here). The B operand of C = A B (B = src) is
 * this set, with kscale folded into A's rows by gwb_oz_split_rows. */
int gwb_oz_split_cols(int32_t s, int64_t krows, int64_t R, const double* src, int64_t ld_src, void* slices,
                      int64_t ldk, int64_t rows_cap, int64_t k0, double* kscale, void* stream);
/* C (M x N float64, row stride ldc) = alpha diag(a_scale) (A B^T) diag(b_scale)
 * + beta C over K columns, for rows a_row0.. of slice set A and b_row0.. of
 * slice set B (b_scale NULL: ones); the s(s+1)/2 slice pairs with
 * i + j <= s + 1 as exact int8 products (int32 accumulation in tensor memory,
 * float64 sums every 8192 columns). Columns K..ceil(K/64)*64-1 of A must be
 * zero. Small tile grids split K, with float64 partials in `work`
 * (gwb_oz_work_bytes; fewer splits with less). A pipeline wait that runs out
 * ORs GWB_ERR_TIMEOUT into *status (device int). */
int64_t gwb_oz_work_bytes(int64_t M, int64_t N, int64_t K);
int gwb_oz_gemm(int32_t s, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, int64_t a_rows_cap,
                int64_t a_row0, const double* a_scale, const void* B, int64_t ldb, int64_t b_rows_cap, int64_t b_row0,
                const double* b_scale, double alpha, double beta, double* C, int64_t ldc, void* work,
                size_t work_bytes, int* status, void* stream);

/* Float64-accurate real products on the int8 tensor cores through residues
 * (the Ozaki scheme's second form: the Chinese remainder theorem). A residue
 * set is n (16, 18 or 20) int8 planes of rows_cap x ldk (ldk a multiple of 64,
 * 16-byte aligned base), plane t at t rows_cap ldk, with one float64 scale
 * per row: row r is scale[r] x_r with x_r an integer vector, |x_r| < 2^p
 * (p = gwb_crt_bits(n): 52, 60, 67), plane t holding x_r mod m_t, centred
 * (m_t = 256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211,
 * 199, 197, 193, 191, 181, 179, 173: the first n). The float64 GEMMs of the
 * Davidson subspace, Ritz, projection and Cholesky-QR steps (gradwave
 * solvers/davidson.py:195-222,428-432,648-657) run on them; the reference
 * has no counterpart.
 *
 * gwb_crt_bits: p for n moduli (-1 for an unsupported n).
 * gwb_crt_constants: the moduli m_t, y_t = (M / m_t)^-1 mod m_t, 1/m_t as a
 * double-double (inv_hi + inv_lo) and M = prod m_t as a double-double
 * (M_hl[0] + M_hl[1]); host only, for inspection and tests. */
int32_t gwb_crt_bits(int32_t n);
int gwb_crt_constants(int32_t n, uint32_t* m, uint32_t* y, double* inv_hi, double* inv_lo, double* M_hl);
/* gwb_crt_split_rows: rows [row0, row0 + rows) of the set from the rows of
 * src (K columns, row stride ld_src), each element times fold[k] when fold is
 * not NULL: scale[row0 + r] = 2^(e - p) with 2^e the power of two above the
 * row's largest magnitude (NaN for a row with a non-finite value), x = the
 * nearest integers to the row / scale; columns K..ldk-1 zeroed. */
int gwb_crt_split_rows(int32_t n, int64_t rows, int64_t K, const double* src, int64_t ld_src, const double* fold,
                       void* planes, int64_t ldk, int64_t rows_cap, int64_t row0, double* scale, void* stream);
/* gwb_crt_split_cols: the transposed layout. src is krows x R (row stride
 * ld_src); row r of the set gets, in columns k0 .. k0 + krows - 1, the
 * residues of the nearest integer to 2^p src[k][r] / kscale[k0 + k], with
 * kscale[k0 + k] the power of two above max_r |src[k][r]| (set here), and
 * scale[r] = 2^-p. The B operand of C = A B (B = src) is this set, with kscale
 * folded into A's rows by gwb_crt_split_rows. */
int gwb_crt_split_cols(int32_t n, int64_t krows, int64_t R, const double* src, int64_t ld_src, void* planes,
                       int64_t ldk, int64_t rows_cap, int64_t k0, double* kscale, double* scale, void* stream);
/* C (M x N float64, row stride ldc) = alpha diag(a_scale) (A B^T) diag(b_scale)
 * + beta C over K <= 2^19 columns, for rows a_row0.. of residue set A and
 * b_row0.. of residue set B: n exact int8 products (int32 sums in tensor
 * memory), each reduced modulo its m_t into a byte of `work`
 * (gwb_crt_work_bytes), then the Chinese remainder reconstruction in
 * double-double. Columns K..ceil(K/64)*64-1 of A must be zero. A pipeline
 * wait that runs out ORs GWB_ERR_TIMEOUT into *status (device int). */
int64_t gwb_crt_work_bytes(int32_t n, int64_t M, int64_t N, int64_t K);
int gwb_crt_gemm(int32_t n, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, int64_t a_rows_cap,
                 int64_t a_row0, const double* a_scale, const void* B, int64_t ldb, int64_t b_rows_cap,
                 int64_t b_row0, const double* b_scale, double alpha, double beta, double* C, int64_t ldc, void* work,
                 size_t work_bytes, int* status, void* stream);

/* Householder tridiagonalisation of a real symmetric m x m matrix across the
 * whole GPU (one cooperative launch, a block per SM, m <= 4096): the
 * reduction step of the subspace eigensolve torch.linalg.eigh (gradwave
 * solvers/davidson.py:66-75,650) for subspaces too large for
 * gwb_heev_lowest. A (column-major, lda; both triangles) is overwritten with
 * LAPACK's dsytrd lower-storage output: d = diag(T), e = the subdiagonal,
 * tau, and reflector j's vector below the subdiagonal of column j
 * (Q = H_0 ... H_{m-2}, H_j = I - tau_j v_j v_j^T, v_j[j+1] = 1). work:
 * gwb_sytrd_work_bytes(m). A grid barrier that waits longer than the
 * gwb_tc_set_wait_limit cycle count ORs GWB_ERR_TIMEOUT into *status. */
size_t gwb_sytrd_work_bytes(int32_t m);
/* Blocks of gwb_sytrd's cooperative launch (0: one per SM): fewer blocks make
 * the grid barrier cheaper and leave less bandwidth for the products. */
int gwb_sytrd_set_blocks(int32_t blocks);
/* The trailing part of gwb_sytrd inside one thread-block cluster: once the
 * trailing matrix fits the cluster's distributed shared memory (about 620
 * rows with 16 CTAs of 1024 threads), a second launch of size x 1 x 1 CTAs
 * finishes the reduction there (two cluster barriers per column instead of
 * two grid barriers). size: -1 the largest cluster the device schedules (16,
 * else 8; the default), 0 the cooperative launch alone, 8 or 16 that size. */
int gwb_sytrd_set_cluster(int32_t size);
/* The middle part of gwb_sytrd across the GPU with the trailing matrix in
 * the shared memory of all SMs (up to ~1790 rows, one 1024-thread CTA per
 * SM, one grid barrier per column), between the panels of the cooperative
 * launch and the cluster: on = 1, or 0 (the default; it measures ~11 us per
 * column, no faster than the cooperative launch). */
int gwb_sytrd_set_grid(int32_t on);
/* Rows of an m x m matrix that gwb_sytrd reduces inside the cluster (0: none). */
int32_t gwb_sytrd_cluster_rows(int32_t m);
/* Phase trace of gwb_sytrd (NULL: off): later launches add the SM cycles of
 * block 0 to cycles10[0..5] = before the product, the product y = A v, the
 * barrier after it, the column's w and the next column's update, the
 * barrier after that, the trailing updates (the cooperative launch); and of
 * the cluster's CTA 0 to cycles10[6..9] = the column and its reflector, the
 * pass over the rows, the exchange, the cluster barrier. For tuning. */
int gwb_sytrd_set_trace(long long* cycles10);
int gwb_sytrd(int32_t m, double* A, int64_t lda, double* d, double* e, double* tau, void* work, size_t work_bytes,
              int* status, void* stream);
/* The nev lowest eigenpairs of a real symmetric m x m matrix (m <= 4096):
 * gwb_sytrd, then multisection on Sturm counts for the eigenvalues of T,
 * inverse iteration for its eigenvectors (clusters within 1e-9 |T|
 * orthogonalised in turn and rotated by a Rayleigh-Ritz of T), Newton-Schulz
 * orthonormalisation and the back-transform U = Q Z in blocks of 256
 * reflectors. A (column-major, lda, both triangles) is overwritten. w: nev
 * ascending; U: m x nev, column-major, ldu. work: gwb_sy_lowest_work_bytes.
 * Replaces torch.linalg.eigh of gradwave solvers/davidson.py:66-75,650 for
 * the lowest Ritz pairs. */
size_t gwb_sy_lowest_work_bytes(int32_t m, int32_t nev);
int gwb_sy_lowest(int32_t m, int32_t nev, double* A, int64_t lda, double* w, double* U, int64_t ldu, void* work,
                  size_t work_bytes, int* status, void* stream);

/* r = hx - eig * x and rn = |r| per (k, band); eig (nk, eig_kstride) float64.
 * Replaces gradwave solvers/davidson.py:656-657. */
int gwb_residual(int32_t nk, int32_t nb, int32_t npw, const void* x, int64_t x_kstride, const void* hx,
                 int64_t hx_kstride, const double* eig, int64_t eig_kstride, void* r, int64_t r_kstride,
                 double* rn, void* stream);

/* out[0] = max rn, out[1] = max over k of #(rn > tol) (device doubles).
 * Replaces the two host reads of gradwave solvers/davidson.py:692,698. */
int gwb_conv_stats(int32_t nk, int32_t nb, const double* rn, double tol, double* out, void* stream);

/* sel (nk, n_add) int32: per k the bands of the n_add largest rn, largest
 * first, ties by band order. Replaces gradwave solvers/davidson.py:729. */
int gwb_select_worst(int32_t nk, int32_t nb, const double* rn, int32_t n_add, int32_t* sel, void* stream);

/* d[k][s] = TPA(t, <x_b|T|x_b>) * r[k][b] / |...| for b = sel[k][s].
 * Replaces gradwave solvers/davidson.py:730-743 and solvers/precond.py:20-39. */
int gwb_precond_teter(int32_t nk, int32_t nb, int32_t n_add, int32_t npw, const void* x, int64_t x_kstride,
                      const void* r, int64_t r_kstride, const double* t, const int32_t* sel, void* d,
                      int64_t d_kstride, void* stream);

/* Insert the new columns m0..m-1 (and mirrored rows) of the subspace matrix
 * S (nk, lds, lds) from C (nk, m, m-m0) = V[:m] . HV[m0:m]^H; Hermitises the
 * new diagonal block. Replaces gradwave solvers/davidson.py:648-649. */
int gwb_subspace_insert(int32_t nk, int32_t m, int32_t m0, const void* C, void* S, int32_t lds,
                        int64_t s_kstride, void* stream);

/* Per k: G (n x n, leading dim ldg) -> lower Cholesky factor in place and
 * Linv = L^-1 (n x n, leading dim n); info[k] = 0 or j+1 at a non-positive
 * pivot j, and bit 1 of *flag is set on any breakdown (flag may be NULL).
 * CholQR step of gradwave solvers/davidson.py:195-222. */
int gwb_chol_inv(int32_t nk, int32_t n, void* G, int32_t ldg, int64_t g_kstride, void* Linv,
                 int64_t linv_kstride, int32_t* info, int32_t* flag, void* stream);

/* Rank repair: rows of D (nk blocks of n rows, d_kstride apart) with norm
 * below thresh are replaced by deterministic noise on the mask (uint8
 * (nk, npw)); bit 0 of *flag is set if any row was repaired. Replaces the
 * jitter of gradwave solvers/davidson.py:450-456. */
int gwb_row_repair(int32_t nk, int32_t n, int32_t npw, void* D, int64_t d_kstride, const uint8_t* mask,
                   double thresh, int32_t* flag, void* stream);

/* Lowest nb eigenpairs of nk Hermitian m x m matrices S (leading dim lds,
 * both triangles filled), float64: eig (nk, nb) ascending, U (nk, m, nb)
 * row-major eigenvector columns; zscratch (nk, gwb_heev_scratch_doubles(m))
 * float64; info[k] = 1 when
 * the QL iteration limit was hit. m <= gwb_heev_max_dim(). One CTA per
 * matrix: Householder tridiagonalisation, Sturm-count multisection for the
 * nb eigenvalues, inverse iteration + CholQR2 + Jacobi Rayleigh-Ritz for the
 * vectors, residual-checked, with implicit QL as the fallback; back-transform.
 * Replaces torch.linalg.eigh in gradwave solvers/davidson.py:66-75,650. */
int gwb_heev_lowest(int32_t nk, int32_t m, int32_t nb, const void* S, int32_t lds, int64_t s_kstride,
                    double* eig, void* U, double* zscratch, int32_t* info, void* stream);
int gwb_heev_max_dim(void);
/* Scratch float64 per matrix that gwb_heev_lowest needs: m * (2m + 8). */
int64_t gwb_heev_scratch_doubles(int32_t m);
/* Diagnostics of gwb_heev_lowest on the current device since load: out[0..3]
 * matrices sent down the QL fallback by reason (pool too small for the
 * bisection path, non-finite inverse iterate, CholQR breakdown, residual
 * above 64 eps |T|), out[4] the bits of the largest residual / |T| the
 * bisection path measured. No counterpart in the reference. */
int gwb_heev_ql_count(unsigned long long* out);

/* gwb_heev_lowest without any device allocation: the caller passes inputs and
 * outputs only, and the eigenvector scratch lives in a fixed 8 MiB device
 * array inside the library (held on every GPU that loads it). For callers
 * whose device memory belongs to a pool allocator or a fixed budget and who
 * therefore cannot call cudaMalloc. No counterpart in the reference.
 * Limits: nk*m*(2m+8) <= 1048576 (else GWB_ERR_ARG); calls share the array, so
 * calls whose kernels may overlap on the GPU race and must be ordered; the
 * first call on a device looks up the array's address and should come before
 * any stream capture. */
int gwb_heev_lowest_noalloc(int32_t nk, int32_t m, int32_t nb, const void* S, int32_t lds, int64_t s_kstride,
                            double* eig, void* U, int32_t* info, void* stream);

/* ======================================================================= */
/* Learned preconditioner (per-plane-wave MLP, BF16, FP32 accumulation).   */
/* No counterpart in the reference: it replaces the TPA coefficient of     */
/* gradwave solvers/precond.py:20-39 by TPA * exp(network), with TPA as    */
/* the per-band fallback. params: float32 master array of                 */
/* gwb_mlp_param_count() values; feats: (n, 4) float32.                   */
/* ======================================================================= */

int gwb_mlp_param_count(void);
/* out[i] = network(feats[i]) (BF16 weights/activations, FP32 accumulation). */
int gwb_mlp_forward(const float* params, int32_t n, const float* feats, float* out, void* stream);
/* grad += d/dparams sum_i w_i (o_i - y_i)^2; loss += the sum (caller zeroes). */
int gwb_mlp_loss_grad(const float* params, int32_t n, const float* feats, const float* target, const float* weight,
                      float* grad, float* loss, void* stream);
/* grad += d/dparams of any loss given dL/do per sample (dout, n floats). */
int gwb_mlp_backward(const float* params, int32_t n, const float* feats, const float* dout, float* grad,
                     void* stream);
/* One Adam step (step >= 1) on the float32 master parameters. */
int gwb_mlp_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr, float beta1,
                 float beta2, float eps, void* stream);
/* Network features of the selected rows at every plane wave: feats (nk, n_add, npw, 4). */
int gwb_precond_features(int32_t nk, int32_t nb, int32_t n_add, int32_t npw, const void* x, int64_t x_kstride,
                         const void* r, int64_t r_kstride, const double* t, const double* eig, const int32_t* sel,
                         float* feats, void* stream);
/* As gwb_precond_teter with the coefficient TPA * exp(clamp(network, -3, 3));
 * bands with tpa_only[k][b] != 0 (uint8 (nk, nb), may be NULL) keep TPA.
 * The network runs on the tcgen05 tensor cores (128 plane waves per MMA
 * tile, accumulators in TMEM), or with gwb_precond_set_kernel(0) on the
 * mma.sync path. work: device scratch of gwb_precond_learned_work_bytes(nk,
 * n_add, npw) bytes (per-row statistics, per-tile partial norms, and in its
 * last 8 bytes an int status that a tensor-core wait which ran out sets to
 * GWB_ERR_TIMEOUT; 8-byte aligned). */
int64_t gwb_precond_learned_work_bytes(int32_t nk, int32_t n_add, int32_t npw);
int gwb_precond_learned(const float* params, int32_t nk, int32_t nb, int32_t n_add, int32_t npw, const void* x,
                        int64_t x_kstride, const void* r, int64_t r_kstride, const double* t, const double* eig,
                        const int32_t* sel, const uint8_t* tpa_only, void* d, int64_t d_kstride, void* work,
                        size_t work_bytes, void* stream);
/* Inference kernel of gwb_precond_learned: 1 tcgen05 (the default), 0 mma.sync. */
int gwb_precond_set_kernel(int32_t which);
/* The learned preconditioner on the Gamma path's embedded real rows (gradwave
 * core/gamma.py:70-160 half-sphere layout): row b of x and r (nb rows,
 * x_row / r_row doubles apart) holds phi with half-sphere coefficient
 * c_G = phi[2G-1] + i phi[2G] (c_0 = phi[0]), G < nhalf. For s < n_add the
 * unit row d[s] (d_row doubles apart; coordinates from 2 nhalf - 1 to npad
 * set to zero) is the preconditioned residual of band sel[s] in the same
 * embedding: TPA * exp(clamp(network, -3, 3)) on the tcgen05 tensor cores
 * (TPA alone when tpa_only[b] != 0; may be NULL). t_half: kinetic diagonal
 * per half-sphere slot; eig: nb. work: gwb_precond_learned_gamma_work_bytes
 * (status int in its last 8 bytes, as above). */
int64_t gwb_precond_learned_gamma_work_bytes(int32_t n_add, int32_t nhalf);
int gwb_precond_learned_gamma(const float* params, int32_t nb, int32_t n_add, int32_t nhalf, int32_t npad,
                              const double* x, int64_t x_row, const double* r, int64_t r_row, const double* t_half,
                              const double* eig, const int32_t* sel, const uint8_t* tpa_only, double* d,
                              int64_t d_row, void* work, size_t work_bytes, void* stream);
/* Stall fallback: count[i] = rounds since rn[i] last fell below ratio * rn_best[i]
 * (rn_best starts at +inf, count at 0); tpa_only[i] = 1 once count[i] >= patience. */
int gwb_stall_update(const double* rn, double* rn_best, uint8_t* count, uint8_t* tpa_only, int32_t n, double ratio,
                     int32_t patience, void* stream);

/* ======================================================================= */
/* Native Davidson driver                                                  */
/* ======================================================================= */

typedef struct {
  int32_t nk, nb, npw;   /* block (nk, nb, npw) with npw = npw_max of the handle */
  int32_t max_dim;       /* basis capacity: min(max_dim_factor * nb, min_k npw), <= gwb_heev_max_dim() */
  int32_t max_iter;
  int32_t mode;          /* 0: float64 applies; 1: float32 expansion applies with float64 certification
                            (the reference's stall rule); 2: as 1, stall rule only near the float32 floor */
  int32_t precond;       /* 0: Teter-Payne-Allan; 1: learned (model = MLP parameters), TPA per-band fallback */
  int32_t flags;         /* bit 0: time every H apply with CUDA events (stats->apply_ms) */
  double tol;            /* residual-norm gate [eV] */
  double t_max;          /* largest kinetic energy of the batch (float32 residual-floor estimate) */
} gwb_davidson_params;

typedef struct {
  int32_t n_iter, hit_max_iter, n_restart, n_cert, n_repair, n_rollback;
  int64_t n_apply_low, n_apply_full;  /* band*k applies in float32 / float64 */
  double max_residual;
  double apply_ms;                    /* device time of the H applies (timing flag only) */
  int64_t n_apply_calls;              /* gwb_ham_apply launches of the solve */
  int64_t n_tpa_fallback;             /* (k, band) pairs the learned preconditioner's stall rule sent to TPA */
} gwb_davidson_stats;

/* Device workspace the solve needs (bytes, 256-byte aligned base). */
int gwb_davidson_workspace_bytes(const gwb_davidson_params* p, size_t* bytes);

/* Lowest nb eigenpairs of the handle's Hamiltonian by batched block Davidson
 * from the start block x0 (complex128, device): eig_out (nk, nb) ascending,
 * vec_out (nk, nb, npw) orthonormal rows with padded slots 0, rn_out (nk, nb)
 * residual norms; stats (HOST) gets the counters. t (nk, npw) kinetic diagonal,
 * mask (nk, npw) uint8. model: float32 network parameters for precond 1
 * (gwb_mlp_param_count values), ignored for precond 0. Returns GWB_OK also
 * when max_iter is hit (stats->hit_max_iter = 1), like the reference.
 * Replaces gradwave solvers/davidson.py:528-774 (davidson_batched) and the
 * registry adapter core of solvers/registry.py:154-182. */
int gwb_davidson_solve(gwb_ham* h, const gwb_davidson_params* p, const void* model, const void* x0,
                       const double* t, const uint8_t* mask, void* workspace, size_t workspace_bytes,
                       double* eig_out, void* vec_out, double* rn_out, gwb_davidson_stats* stats, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GWB_H_ */
