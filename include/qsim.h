/*
 * qsim.h -- C-ABI of libqsim.so, the sm_100a gate-application library behind
 * quict_b200's StateVectorSimulator / DensityMatrixSimulator.
 *
 * Conventions shared by every entry point
 * ---------------------------------------
 *  - A state vector is a contiguous device array of 2^n complex numbers,
 *    interleaved (re, im), in complex64 (QS_C64) or complex128 (QS_C128).
 *  - "bit" always means a VECTOR bit: amplitude index i has bit b set iff
 *    (i >> b) & 1.  A QuICT qubit q of an n-qubit circuit is vector bit n-1-q
 *    (QuICT/core/qubit/qubit.py:192-213, statevector_simulator.py:170-172).
 *  - A k-qubit matrix is row-major 2^k x 2^k; matrix-index bit (k-1-j)
 *    belongs to the j-th listed vector bit ("big-endian over the argument
 *    list", QuICT/core/utils/utils.py:8-56).
 *  - Host matrices are passed as complex128 (double re, im pairs) and are
 *    rounded to the state's precision inside the call, the same rounding as
 *    numpy's astype(complex64) that QuICT applies (gate.py:945-951).
 *  - The caller owns every buffer.  The library never allocates device
 *    memory; scratch comes from a caller workspace whose size the matching
 *    *_ws_bytes() query returns.
 *  - Every call is stream-ordered on `stream` (a cudaStream_t; NULL = legacy
 *    default stream), performs no implicit device synchronisation and returns
 *    QS_OK or a negative QS_E* code.  qs_last_error() returns a thread-local
 *    description of the last failure.  No C++ exception crosses the ABI.
 *
 * The reference (taofei95/quict) dispatches one CuPy RawKernel per gate from
 * Python through LinAlgLoader (QuICT/ops/utils/algorithm_loader.py:17-54);
 * each entry point below names the reference interface it replaces.
 */
#ifndef QSIM_H
#define QSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define QS_OK          0
#define QS_EINVAL     -1   /* bad argument (qubit out of range, bad kind ...) */
#define QS_ECUDA      -2   /* CUDA launch / runtime error                      */
#define QS_EWORKSPACE -3   /* caller workspace too small                       */
#define QS_ENOTSUP    -4   /* valid but unsupported configuration              */
#define QS_ETIMEOUT   -5   /* a bounded device-side wait gave up               */

/* ---- dtypes ------------------------------------------------------------ */
#define QS_C64   0
#define QS_C128  1

/* ---- single-gate kinds (qs_apply_1q / qs_apply_2q) ----------------------- */
#define QS_K_DENSE     0  /* full matrix                                       */
#define QS_K_DIAG      1  /* diagonal; a leading 1 on the diagonal is skipped  */
#define QS_K_ANTIDIAG  2  /* 1q only: v0' = m01*v1, v1' = m10*v0 (X, Y, CX ...) */
#define QS_K_SWAP      3  /* 2q only: v01' = m12*v10, v10' = m21*v01, v00*=m00, v11*=m33 */

/* ---- fused-pass op kinds ------------------------------------------------- */
#define QS_OP_MAT   1     /* dense 2^m x 2^m on m tile-resident bits           */
#define QS_OP_DIAG  2     /* diagonal on m bits anywhere in the vector         */
#define QS_OP_ANTI  3     /* m = 1: anti-diagonal 2x2 (entries m01, m10 used)   */
#define QS_OP_SWAP  4     /* m = 2: swap-like 4x4 (m00, m12, m21, m33 used)     */
#define QS_OP_EXPECT 5    /* qs_adjoint_fused only: partial <lam| G |psi> over the
                             tile for a generator G (m <= 2, dense, or diagonal
                             with QS_OPF_DIAG), summed into partials[slot]     */
#define QS_MAX_PASS_MATS 2048  /* matrix entries one pass may reference        */
#define QS_OPF_UNIT 1     /* ANTI: m01 = m10 = 1; SWAP: m00 = m12 = m21 = m33 = 1 */
#define QS_OPF_DIAG 2     /* EXPECT: the generator is diagonal (2^m entries)   */

/* ---- probability sources and sampling modes ------------------------------ */
#define QS_SRC_SV  0      /* p_i = |vec[i]|^2                                  */
#define QS_SRC_DM  1      /* p_i = Re rho[i, i] of a 2^n x 2^n density matrix  */
#define QS_SAMPLE_CDF  0  /* one uniform per shot: smallest i with
                             u * total <= CDF[i] (FP64, unnormalised CDF);
                             indices of probability 0 are never returned    */
#define QS_SAMPLE_SEQ  1  /* n uniforms per shot, qubit 0 (MSB) first, outcome
                             1 iff u > P(0) -- the reference's per-qubit rule  */

#define QS_MAX_TILE_BITS 14
#define QS_MAX_PASS_OPS  160

/* One op of a fused pass.  80 bytes, plain old data (mirrored by ctypes). */
typedef struct qs_op {
    int32_t  kind;       /* QS_OP_MAT, QS_OP_DIAG, QS_OP_ANTI or QS_OP_SWAP     */
    int32_t  m;          /* number of target bits, 1..4                         */
    int32_t  tgt[4];     /* tile-local position of target j, or -1 when the bit
                            lies outside the tile (allowed for QS_OP_DIAG only) */
    int32_t  gbit[4];    /* vector bit of target j (matrix-index bit m-1-j)     */
    uint32_t lctrl;      /* control mask on tile-local positions                */
    uint32_t flags;      /* QS_OPF_* hints about the matrix entries             */
    uint64_t gctrl;      /* control mask on vector bits outside the tile        */
    int64_t  mat;        /* element offset of the op's matrix in the table
                            (QS_OP_DIAG: 2^m entries, the other kinds: 4^m)    */
    int64_t  mat_stride; /* batched passes: instance i uses mat + i*mat_stride  */
    int32_t  slot;       /* QS_OP_EXPECT: output slot                          */
    int32_t  pad1;
} qs_op;

/* One fused pass: a tile of 2^k amplitudes made of vector bits 0..nlow-1 and
 * hi[0..k-nlow-1] (ascending), and ops [op_begin, op_begin+op_count).
 * Batched state (inst_shift > 0): the vector holds instances of 2^inst_shift
 * amplitudes; instance = index >> inst_shift (with the pair bit cleared).
 * All tile bits other than the pair bit must be below inst_shift, so a tile
 * belongs to one instance.
 * pair: 0, or b + 1 where vector bit b separates psi (0) from lam (1) in the
 * combined vector of qs_adjoint_pair; b must be a tile bit of every pass
 * that has EXPECT ops. */
typedef struct qs_pass {
    int32_t k;
    int32_t nlow;
    int32_t hi[QS_MAX_TILE_BITS];
    int32_t op_begin;
    int32_t op_count;
    int32_t inst_shift;
    int32_t pair;
} qs_pass;

/* ---- library ------------------------------------------------------------ */
int         qs_version(void);
const char* qs_last_error(void);
/* Number of SMs of the current device (grid sizing; host query only). */
int         qs_device_sm_count(void);

/* ---- state preparation -------------------------------------------------- */
/* vec <- |0...0> (replaces initial_state_vector, statevector_simulator.py:115-121). */
int qs_init_zero(void* vec, int n, int dtype, void* stream);
/* vec *= (re + i*im) (replaces float_multiply / complex_multiply,
 * QuICT/ops/gate_kernel/multigpu_gate_func.py:13-102). */
int qs_scale(void* vec, int n, int dtype, double re, double im, void* stream);

/* ---- single gates --------------------------------------------------------- */
/* One-target gate on `bit`, applied where all `ctrl_mask` bits are 1.
 * mat: host complex128[4] (row-major 2x2).  Replaces, by kind:
 *   DENSE    normal_targ, normal_ctargs           gate_function.py:1095-1119, 1236-1262
 *   DIAG     diagonal_targ, control_targ, diagonal_ctargs, control_ctargs,
 *            diagonal_more                         gate_function.py:1034-1058, 1151-1233, 1517-1552
 *   ANTIDIAG swap_targ, reverse_targ, reverse_ctargs, reverse_more
 *                                                  gate_function.py:1362-1442, 1479-1514 */
int qs_apply_1q(void* vec, int n, int dtype, int bit, uint64_t ctrl_mask,
                int kind, const double* mat, void* stream);

/* Two-target gate; bit_hi carries matrix-index bit 1 (first argument), bit_lo
 * matrix-index bit 0.  mat: host complex128[16].  Replaces
 *   DENSE normal_targs, ctrl_normal_targs, normal_normal_targs,
 *         diagonal_normal_targs                    gate_function.py:1122-1148, 1265-1359
 *   DIAG  diagonal_targs                           gate_function.py:1061-1092
 *   SWAP  swap_targs, swap_tmore                   gate_function.py:1445-1476, 1555-1590 */
int qs_apply_2q(void* vec, int n, int dtype, int bit_hi, int bit_lo,
                uint64_t ctrl_mask, int kind, const double* mat, void* stream);

/* Dense k-target gate, 1 <= k <= 10, in place.  bits[j] carries matrix-index
 * bit k-1-j.  mat_dev: DEVICE complex128[4^k].  Replaces matrix_dot_vector
 * (QuICT/ops/linalg/gpu_calculator.py:343-478), which is out of place. */
int qs_apply_kq(void* vec, int n, int dtype, int k, const int32_t* bits,
                uint64_t ctrl_mask, const void* mat_dev, void* stream);

/* ---- fused passes ---------------------------------------------------------- */
/* Applies `npasses` passes; each pass is one launch that streams the vector
 * through shared-memory tiles once and applies all of its ops per tile.
 * passes / ops: HOST arrays (nops_total entries in ops); mats_dev: DEVICE
 * table of mats_count complex entries in the state's dtype.  Every pass and op
 * is validated on the host before the first launch.
 * No reference counterpart: the reference launches one kernel per gate
 * (statevector_simulator.py:155-164). */
int qs_apply_fused(void* vec, int n, int dtype, const qs_pass* passes, int npasses,
                   const qs_op* ops, int64_t nops_total, const void* mats_dev,
                   int64_t mats_count, void* stream);

/* qs_apply_fused with the matrix table also given in HOST memory (the same
 * values as mats_dev, in the state's precision).  A register pass then runs
 * as a kernel generated for that pass alone and compiled at run time
 * (NVRTC, sm_100a) when the library's JIT mode allows it: its ops, slot
 * masks and relayout addresses are constants of the code, plain exchanges
 * are register renamings, and its matrices travel in the launch's parameter
 * block (read as constant-bank operands).  Compiled kernels are cached by
 * their source, which depends on the pass's structure and on which matrix
 * entries are exactly 0, 1 or -1, not on the other values.  Until a pass's
 * kernel is compiled (mode QS_JIT_ASYNC) the generic kernel runs it, with
 * the same results.  mats_host may be NULL (the generic kernels only).
 * No counterpart in the reference, which launches one kernel per gate. */
int qs_apply_fused_ex(void* vec, int n, int dtype, const qs_pass* passes, int npasses,
                      const qs_op* ops, int64_t nops_total, const void* mats_dev,
                      const void* mats_host, int64_t mats_count, void* stream);

/* qs_adjoint_pair with the matrix table also in HOST memory (as
 * qs_apply_fused_ex): pair passes then run as generated kernels when the
 * JIT mode allows it, with per-instance tables staged in shared memory. */
int qs_adjoint_pair_ex(void* psilam, int n, int dtype, const qs_pass* passes, int npasses,
                       const qs_op* ops, int64_t nops_total, const void* mats_dev,
                       const void* mats_host, int64_t mats_count, double* partials_dev,
                       int64_t partials_count, void* stream);

/* ---- run-time compiled passes ------------------------------------------------ */
#define QS_JIT_OFF   0    /* generic fused kernels only                             */
#define QS_JIT_ASYNC 1    /* compile on host threads; generic kernels meanwhile (default;
                             the QS_JIT environment variable sets the initial mode) */
#define QS_JIT_SYNC  2    /* compile before the first launch of a new pass shape    */
/* Set the mode; returns the previous one (or a negative error). */
int qs_jit_set_mode(int mode);
/* Wait until no compilation is queued or running (timeout_s < 0: no limit);
 * QS_ETIMEOUT when the limit passes first. */
int qs_jit_wait(double timeout_s);
/* out[0..n-1] <- kernels compiled, compilations failed, compilations pending,
 * launches of compiled kernels, launches that ran the generic kernel while a
 * compilation was pending, total compile milliseconds, cache hits. */
int qs_jit_stats(int64_t* out, int n);
/* Drop queued compilations and wait for the running ones to finish (call
 * before the process exits while compilations may be running; passes not yet
 * compiled keep running on the generic kernels). */
int qs_jit_shutdown(void);
/* Log of the last failed compilation or load ("" if none). */
const char* qs_jit_last_log(void);
/* Compile `src` with NVRTC only (no device needed); *cubin_bytes <- size. */
int qs_jit_compile_check(const char* src, int64_t* cubin_bytes);
/* The generated source of launch `launch_index` of one register pass (as
 * qs_apply_fused_ex would plan it), without a device: *src_len <- its
 * length; up to out_size - 1 bytes are copied to `out` (may be NULL).
 * QS_ENOTSUP for passes that do not run as generated kernels. */
int qs_jit_pass_source(int n, int dtype, const qs_pass* pass, const qs_op* ops, int64_t nops_total,
                       const void* mats_host, int64_t mats_count, int launch_index, char* out,
                       size_t out_size, int64_t* src_len);

/* ---- differentiation / observables ---------------------------------------- */
/* Backward-sweep pass of the adjoint method: every QS_OP_MAT / DIAG / ANTI /
 * SWAP op is applied to BOTH psi and lam (the caller passes the inverse
 * gates), and every QS_OP_EXPECT op adds the tile's partial sum of
 * conj(lam_i) (G psi)_i to partials[2 * (slot * ntiles + tile)] (re, im; FP64),
 * ntiles = 2^(n - k) of the pass.  partials_count bounds the slots*ntiles.
 * Replaces per-parameter circuit re-runs (parameter shift); the reference has
 * no gradient path (its ML package is not part of it). */
int qs_adjoint_fused(void* psi, void* lam, int n, int dtype, const qs_pass* passes, int npasses,
                     const qs_op* ops, int64_t nops_total, const void* mats_dev, int64_t mats_count,
                     double* partials_dev, int64_t partials_count, void* stream);

/* The same backward sweep on ONE vector of 2^n amplitudes holding psi in the
 * half where bit b = pair - 1 is 0 and lam in the other half (every pass sets
 * `pair`, and passes with EXPECT ops keep bit b in their tile; with
 * instances, b is the top bit).  Ops
 * on the other bits act on both halves at once, and the register-tile kernel
 * keeps each psi amplitude beside its lam partner, so EXPECT ops run on chip
 * between the gates.  partials: as for qs_adjoint_fused, ntiles = 2^(n - k).
 * Needs register tiles: k in [9, 12] (complex128) or [10, 13] (complex64),
 * nlow >= 5; dense ops act on at most 2 bits.  Replaces the same per-parameter re-runs as qs_adjoint_fused. */
int qs_adjoint_pair(void* psilam, int n, int dtype, const qs_pass* passes, int npasses,
                    const qs_op* ops, int64_t nops_total, const void* mats_dev, int64_t mats_count,
                    double* partials_dev, int64_t partials_count, void* stream);

/* out = sum_t c_t P_t psi for Pauli strings P_t = i^popc(x&z) X^x Z^z (x, z:
 * HOST arrays of masks over vector bits, coeff: HOST complex128 pairs).  out
 * and psi must not alias.  Used for lam = H psi. */
int qs_apply_pauli_sum(const void* psi, void* out, int n, int dtype, const uint64_t* xmask,
                       const uint64_t* zmask, const double* coeff, int nterms, void* stream);

/* out_dev[2*i] + i*out_dev[2*i+1] = sum over instance i of conj(a_j) b_j
 * (FP64), instances of 2^inst_bits amplitudes.  ws: at least 16 bytes per
 * instance; a larger workspace (up to 16 KiB per instance) lets each
 * instance use more thread blocks (partial sums). */
int qs_inner_batched(const void* a, const void* b, int n, int dtype, int inst_bits, double* out_dev,
                     void* ws, size_t ws_bytes, void* stream);

/* out[s] = sum_{t < seglen} in[s * seglen + t] for complex FP64 pairs. */
int qs_segment_sum(const double* in_dev, int64_t nseg, int64_t seglen, double* out_dev, void* stream);

/* ---- persistent batch: many problems in one launch ------------------------- */
/* One problem of a batch: an n-qubit circuit from |0...0>, its observable H
 * and the adjoint sweep of its gradient.  Passes, ops, matrices, observable
 * terms and weights index arrays shared by the whole batch. */
typedef struct qs_batch_inst {
  int32_t n;           /* qubits; psi has 2^n amplitudes                       */
  int32_t fwd_begin;   /* forward passes[fwd_begin, +nfwd) over n bits; the    */
  int32_t nfwd;        /*   first reads |0...0> (>= 1 pass)                    */
  int32_t bwd_begin;   /* backward pair passes[bwd_begin, +nbwd) over n + 1    */
  int32_t nbwd;        /*   bits, pair = n + 1 (psi / lam on vector bit n)      */
  int32_t term_begin;  /* H = sum of terms [term_begin, +nterms) (1..128) of    */
  int32_t nterms;      /*   xmask / zmask / coeff (as qs_apply_pauli_sum)       */
  int32_t nslots;      /* EXPECT slots of the backward passes                  */
  int32_t nparams;     /* gradient length                                       */
  int32_t pad;
  int64_t w_begin;     /* W = weights[w_begin, +nparams*nslots), row-major:    */
                       /*   gradient = W Im(per-slot sums of <lam|G|psi>)       */
} qs_batch_inst;

/* What a planned batch needs (filled by qs_batch_plan). */
typedef struct qs_batch_sizes {
  int64_t blob_bytes;       /* the plan (copy it to the device unchanged)       */
  int64_t state_elems;      /* state pool: complex elements (sum of 2^(n+1))    */
  int64_t partial_doubles;  /* partials pool                                     */
  int64_t grad_doubles;     /* gradient output: instances' gradients in order   */
  int64_t energy_doubles;   /* energy output: (re, im) per instance             */
  int64_t ctrl_bytes;       /* control words                                     */
  int64_t smem_bytes;       /* dynamic shared memory per CTA                     */
  int32_t threads;          /* CTA size                                          */
  int32_t nitems;           /* work items                                        */
  int32_t nstages;          /* register stages over all instances                */
  int32_t big;              /* some pass needs the wide dense-op code paths      */
  int32_t dtype;
  int32_t jit_fns;          /* generated register-stage functions (see below)   */
  uint64_t jit_key;         /* identifies them for qs_batch_launch               */
} qs_batch_sizes;

/* Plan a batch on the host.  Every stage of every problem (register passes,
 * lam = H psi with the energy partials, the final reduction) is cut into
 * work items of `tiles_per_item` tiles / `amps_per_ham_item` amplitudes.
 * mats_host (the matrix table in HOST memory, the state's precision; may be
 * NULL): the register stages of problems with at least jit_min_qubits
 * qubits are also generated as straight-line device functions (as
 * qs_apply_fused_ex generates kernels), queued for compilation (NVRTC,
 * relocatable) when the plan is written, and linked with the batch kernel
 * (nvJitLink) at the first qs_batch_launch that finds them compiled.
 * blob == NULL: only fill *sizes (and state_off[i], the element offset of
 * problem i's pair vector in the state pool, if state_off != NULL); else
 * write the plan (blob_bytes >= sizes->blob_bytes).  Passes follow the rules
 * of qs_apply_fused / qs_adjoint_pair and must be register tiles (k in
 * [9, 12] complex128 / [10, 13] complex64, nlow >= 5); a problem's backward
 * passes share one k.  No reference counterpart (the reference has neither
 * gradients nor batching). */
int qs_batch_plan(int dtype, const qs_batch_inst* inst, int ninst, const qs_pass* passes, int npasses,
                  const qs_op* ops, int64_t nops, int64_t mats_count, const void* mats_host,
                  int jit_min_qubits, const uint64_t* xmask,
                  const uint64_t* zmask, const double* coeff, int nterms_total, const double* weights,
                  int64_t nweights, int64_t tiles_per_item, int64_t amps_per_ham_item, void* blob,
                  size_t blob_bytes, qs_batch_sizes* sizes, int64_t* state_off);

/* Compile and link the generated functions of a plan with the batch kernel
 * (waiting for their compilation) without loading the result: no device is
 * needed.  *cubin_bytes <- the linked cubin's size (0 for a plan without
 * generated functions).  QS_ENOTSUP with the compiler's or linker's message
 * when a step fails. */
int qs_batch_link_check(const qs_batch_sizes* sizes, int64_t* cubin_bytes);

/* Run a planned batch as ONE persistent kernel launch (after a memset of the
 * control words, both on `stream`).  blob_dev: the plan in device memory
 * (16-byte aligned); states: the state pool; mats: the matrix table the ops
 * index (mats_count entries, the state's dtype); partials, energies (re, im
 * per problem), grads: outputs sized by qs_batch_plan; ctrl: ctrl_bytes of
 * device memory.  Work items wait for their problem's earlier stages with a
 * bounded wait of timeout_s seconds; a wait that gives up stores
 * (1 << 32) | item in control word 1 (bytes 8..15 of ctrl, 0 on success) and
 * the launch ends early.  A plan with generated functions runs as the
 * linked kernel once it is linked on this device (returns 1), else as the
 * generic kernel (returns QS_OK), with the same results up to rounding;
 * during stream capture nothing is compiled or linked, so warm up first.
 * Replaces nothing in the reference (see above). */
int qs_batch_launch(const qs_batch_sizes* sizes, const void* blob_dev, void* states, const void* mats,
                    double* partials, double* energies, double* grads, void* ctrl, size_t ctrl_bytes,
                    double timeout_s, void* stream);

/* ---- measurement, reset, sampling ------------------------------------------ */
size_t qs_reduce_ws_bytes(int n);
/* *out_dev <- sum over {i : bit b of i is 0} of p_i, in FP64 (src = QS_SRC_*).
 * Replaces measured_prob_calculate (gate_function.py:1751-1776). */
int qs_prob0(const void* src, int n, int dtype, int src_kind, int bit,
             void* ws, size_t ws_bytes, double* out_dev, void* stream);
/* *out_dev <- sum_i p_i in FP64. */
int qs_norm2(const void* src, int n, int dtype, int src_kind,
             void* ws, size_t ws_bytes, double* out_dev, void* stream);
/* Keep the `outcome` half of `bit`, scale it by `scale`, zero the other half.
 * Replaces apply_measuregate's collapse (gate_function.py:1779-1815). */
int qs_collapse(void* vec, int n, int dtype, int bit, int outcome, double scale, void* stream);
/* Reset `bit` to |0> given P(0) = p0, with the reference's rule
 * (gate_function.py:1818-1847; cpu_calculator.py:366-384). */
int qs_reset(void* vec, int n, int dtype, int bit, double p0, void* stream);

/* Sampling workspace: a sum tree of FP64 block sums. */
size_t qs_sample_ws_bytes(int n);
int qs_sample_prepare(const void* src, int n, int dtype, int src_kind,
                      void* ws, size_t ws_bytes, void* stream);
/* out_idx_dev[s] <- sampled basis index of shot s.  u_dev: DEVICE doubles,
 * `shots` of them (QS_SAMPLE_CDF) or shots*n (QS_SAMPLE_SEQ, shot-major).
 * Replaces the shots x qubits loop of StateVectorSimulator.sample
 * (statevector_simulator.py:595-626). */
int qs_sample(const void* src, int n, int dtype, int src_kind, const void* ws,
              size_t ws_bytes, const double* u_dev, int64_t shots, int mode,
              int64_t* out_idx_dev, void* stream);
/* Allocation-free variant of qs_sample_prepare + qs_sample.  No counterpart
 * in the reference.  It exists for callers that cannot allocate device
 * memory: a process whose device memory is already handed out to its own
 * pool allocator (so an extra cudaMalloc can fail or fragment it), or a
 * C / FFI caller that owns only the state, the uniforms and the output and
 * has nowhere to keep a workspace.  The FP64 sum tree lives in a file-scope
 * device array of the library (1 MiB on every device that loads it, held until
 * the process exits), so the call allocates nothing and frees nothing.
 * Limit: n <= QS_NOALLOC_SAMPLE_MAX_QUBITS (26); larger n returns QS_EINVAL.
 * Each call made outside stream capture looks up the array's device address
 * on the current device (cudaGetSymbolAddress, with that device current), so
 * a context rebuilt by cudaDeviceReset is handled; a call inside a capture
 * reuses the address the last call outside one found, so make the first
 * call on each device before any stream capture begins.  All calls share the one array and it
 * keeps the last call's contents (each call overwrites every node it reads),
 * so calls whose work overlaps on the GPU -- e.g. on two streams -- race:
 * order them on one stream.  Arguments and results as qs_sample. */
#define QS_NOALLOC_SAMPLE_MAX_QUBITS 26
int qs_sample_noalloc(const void* src, int n, int dtype, int src_kind, const double* u_dev,
                      int64_t shots, int mode, int64_t* out_idx_dev, void* stream);

/* counts_dev[idx_dev[s]] += 1 (int64, caller zeroes counts_dev). */
int qs_histogram(const int64_t* idx_dev, int64_t shots, int64_t* counts_dev,
                 int64_t ncounts, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QSIM_H */
