/*
 * nqpu_b200.h — C ABI of the B200 statevector engine.
 *
 * The first block of declarations is the drop-in boundary: the same names,
 * argument meaning, ownership rules and error codes as the reference's C FFI
 * (sdk/rust/src/infra/bindings/c_ffi.rs, header text at c_ffi.rs:1480-1620),
 * so a caller linking against the reference's generated `nqpu_metal.h` can link
 * this library instead.  Each declaration cites the reference entry point it
 * replaces.  Amplitudes live in B200 HBM; every call runs hand-written sm_100a
 * kernels on the state's own CUDA stream.  There is no CPU fallback: when no
 * CUDA device is usable, creation returns NULL and every other call returns
 * NQPU_SIMULATION_FAILED.
 *
 * The second block holds additions in the same conventions (opaque handles,
 * NqpuError returns, caller-owned output buffers with explicit lengths): the
 * complex64 state, the extended gate set, whole-register reductions, the fused
 * (tensor-core) execution mode, batched execution and the request server.
 *
 * Threading: a handle is used by one host thread at a time (the reference's
 * `&mut` aliasing contract, c_ffi.rs:620-650).  The RNG used by measurement and
 * sampling is thread-local and seeded by nqpu_set_seed, as in c_ffi.rs:49-66.
 */
#ifndef NQPU_B200_H
#define NQPU_B200_H

#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Types (c_ffi.rs:76-204)                                             */
/* ------------------------------------------------------------------ */

typedef struct NqpuState NqpuState;       /* c_ffi.rs:76  opaque state      */
typedef struct NqpuCircuit NqpuCircuit;   /* c_ffi.rs:85  opaque circuit    */

typedef enum {                            /* c_ffi.rs:97-113                */
    NQPU_OK                = 0,
    NQPU_INVALID_QUBIT     = 1,
    NQPU_INVALID_PARAMETER = 2,
    NQPU_ALLOCATION_FAILED = 3,
    NQPU_SIMULATION_FAILED = 4,
    NQPU_NULL_POINTER      = 5,
    NQPU_INVALID_HANDLE    = 6
} NqpuError;

typedef struct { double re; double im; } NqpuComplex;          /* c_ffi.rs:121 */
typedef struct { uint32_t outcome; double probability; } NqpuMeasurement; /* :178 */
typedef struct {                                                 /* c_ffi.rs:188 */
    uint32_t num_qubits;
    uint64_t seed;
    bool     use_gpu;
    uint32_t num_threads;
} NqpuConfig;
typedef struct { uint32_t major; uint32_t minor; uint32_t patch; } NqpuVersion; /* :197 */

/* ------------------------------------------------------------------ */
/* State management                                                    */
/* ------------------------------------------------------------------ */

/* c_ffi.rs:789  complex128 state |0..0>; NULL if n==0, n>30 or no device. */
NqpuState*  nqpu_state_create(uint32_t num_qubits);
/* c_ffi.rs:805  NULL-safe. */
void        nqpu_state_destroy(NqpuState* state);
/* c_ffi.rs:817  device-to-device deep copy; NULL on NULL input or OOM. */
NqpuState*  nqpu_state_clone(const NqpuState* state);
/* c_ffi.rs:836  0 on NULL. */
uint32_t    nqpu_state_num_qubits(const NqpuState* state);
/* c_ffi.rs:850  index >= 2^n -> NQPU_INVALID_PARAMETER. */
NqpuError   nqpu_state_get_amplitude(const NqpuState* state, uint64_t index, NqpuComplex* out);
/* c_ffi.rs:877  does not renormalise. */
NqpuError   nqpu_state_set_amplitude(NqpuState* state, uint64_t index, NqpuComplex amp);
/* c_ffi.rs:900  len must be >= 2^n. */
NqpuError   nqpu_state_probabilities(const NqpuState* state, double* out, uint64_t len);
/* c_ffi.rs:929  squared norm (FP64 reduction); -1.0 on NULL. */
double      nqpu_state_norm(const NqpuState* state);
/* c_ffi.rs:941 */
NqpuError   nqpu_state_reset(NqpuState* state);

/* ------------------------------------------------------------------ */
/* Gate operations (c_ffi.rs:956-1140), one kernel launch per gate     */
/* ------------------------------------------------------------------ */

NqpuError   nqpu_gate_h(NqpuState* state, uint32_t qubit);           /* c_ffi.rs:995  */
NqpuError   nqpu_gate_x(NqpuState* state, uint32_t qubit);           /* c_ffi.rs:996  */
NqpuError   nqpu_gate_y(NqpuState* state, uint32_t qubit);           /* c_ffi.rs:997  */
NqpuError   nqpu_gate_z(NqpuState* state, uint32_t qubit);           /* c_ffi.rs:998  */
NqpuError   nqpu_gate_s(NqpuState* state, uint32_t qubit);           /* c_ffi.rs:999  */
NqpuError   nqpu_gate_t(NqpuState* state, uint32_t qubit);           /* c_ffi.rs:1000 */
NqpuError   nqpu_gate_rx(NqpuState* state, uint32_t qubit, double angle); /* c_ffi.rs:1002 */
NqpuError   nqpu_gate_ry(NqpuState* state, uint32_t qubit, double angle); /* c_ffi.rs:1003 */
NqpuError   nqpu_gate_rz(NqpuState* state, uint32_t qubit, double angle); /* c_ffi.rs:1004 */
NqpuError   nqpu_gate_cx(NqpuState* state, uint32_t control, uint32_t target); /* c_ffi.rs:1010 */
NqpuError   nqpu_gate_cz(NqpuState* state, uint32_t control, uint32_t target); /* c_ffi.rs:1032 */
NqpuError   nqpu_gate_swap(NqpuState* state, uint32_t q1, uint32_t q2);       /* c_ffi.rs:1054 */
/* c_ffi.rs:1079  row-major [[m00,m01],[m10,m11]]. */
NqpuError   nqpu_gate_custom_1q(NqpuState* state, uint32_t qubit, const NqpuComplex* matrix);
/* c_ffi.rs:1111  row-major 4x4; basis |q1 q2>, q1 is the HIGH bit of the sub-index. */
NqpuError   nqpu_gate_custom_2q(NqpuState* state, uint32_t q1, uint32_t q2, const NqpuComplex* matrix);

/* ------------------------------------------------------------------ */
/* Measurement (c_ffi.rs:1151-1250)                                    */
/* ------------------------------------------------------------------ */

/* c_ffi.rs:1151  collapse; r drawn from the thread-local xorshift64*. */
NqpuError   nqpu_measure(NqpuState* state, uint32_t qubit, NqpuMeasurement* out);
/* c_ffi.rs:1177  qubits measured 0..n-1 in order. */
NqpuError   nqpu_measure_all(NqpuState* state, uint32_t* out, uint32_t num_qubits);
/* c_ffi.rs:1205 */
NqpuError   nqpu_expectation_z(const NqpuState* state, uint32_t qubit, double* out);
/* c_ffi.rs:1231  outcome = first i with r < cumsum_i (else 2^n-1). */
NqpuError   nqpu_sample(const NqpuState* state, uint32_t num_shots, uint64_t* out);

/* ------------------------------------------------------------------ */
/* Circuit API (c_ffi.rs:1259-1400)                                    */
/* ------------------------------------------------------------------ */

NqpuCircuit* nqpu_circuit_create(uint32_t num_qubits);            /* c_ffi.rs:1259 */
void         nqpu_circuit_destroy(NqpuCircuit* circuit);          /* c_ffi.rs:1273 */
NqpuError    nqpu_circuit_add_h(NqpuCircuit* circuit, uint32_t qubit);                 /* :1283 */
NqpuError    nqpu_circuit_add_cx(NqpuCircuit* circuit, uint32_t control, uint32_t target); /* :1300 */
NqpuError    nqpu_circuit_add_rx(NqpuCircuit* circuit, uint32_t qubit, double angle);  /* :1322 */
/* c_ffi.rs:1346  runs the circuit through the tiled multi-gate pass engine. */
NqpuError    nqpu_circuit_execute(const NqpuCircuit* circuit, NqpuState* state);
uint32_t     nqpu_circuit_gate_count(const NqpuCircuit* circuit); /* c_ffi.rs:1372 */
uint32_t     nqpu_circuit_depth(const NqpuCircuit* circuit);      /* c_ffi.rs:1385 */

/* ------------------------------------------------------------------ */
/* Utility (c_ffi.rs:1403-1470)                                        */
/* ------------------------------------------------------------------ */

NqpuVersion  nqpu_version(void);                    /* c_ffi.rs:1403 */
const char*  nqpu_error_message(NqpuError error);   /* c_ffi.rs:1426 */
void         nqpu_set_seed(uint64_t seed);          /* c_ffi.rs:1444 */
void         nqpu_set_num_threads(uint32_t threads);/* c_ffi.rs:1460 accepted, no effect on GPU */

/* ================================================================== */
/* Additions (same conventions)                                         */
/* ================================================================== */

typedef enum { NQPU_C128 = 0, NQPU_C64 = 1 } NqpuDtype;

/* Engine modes for nqpu_circuit_execute_ex. */
typedef enum {
    NQPU_MODE_TILED   = 0,  /* multi-gate smem/register tiled passes (default)       */
    NQPU_MODE_PERGATE = 1,  /* one full-state kernel launch per gate (plain per-gate) */
    NQPU_MODE_FUSED   = 2,  /* <=5-qubit fusion, split-TF32 tcgen05 contractions      */
    NQPU_MODE_TENSOR  = 3,  /* complex64, n >= 12: up to 3 fused 5-qubit unitaries per
                               HBM pass, split-FP16 tcgen05 GEMMs on a shared-memory tile */
    NQPU_MODE_AUTO    = 4   /* per gate run between mid-circuit measurements: the tensor
                               mode when its modelled device time is lower, else tiled */
} NqpuMode;

/* Like nqpu_state_create with a dtype; 1 <= n <= 34 (HBM-bounded). */
NqpuState*  nqpu_state_create_ex(uint32_t num_qubits, NqpuDtype dtype);
NqpuDtype   nqpu_state_dtype(const NqpuState* state);
/* Set the state to the computational basis state |index>. */
NqpuError   nqpu_state_set_basis(NqpuState* state, uint64_t index);
/* Copy all 2^n amplitudes to the host as complex128 (len >= 2^n). */
NqpuError   nqpu_state_get_amplitudes(const NqpuState* state, NqpuComplex* out, uint64_t len);
/* Load all 2^n amplitudes from the host (rounded to the state's dtype). */
NqpuError   nqpu_state_set_amplitudes(NqpuState* state, const NqpuComplex* in, uint64_t len);
/* Block until all work queued on the state's stream has finished. */
NqpuError   nqpu_state_synchronize(const NqpuState* state);
/* The cudaStream_t the state's work is queued on (for CUDA-event timing). */
void*       nqpu_state_cuda_stream(const NqpuState* state);

/* Reference GateOperations coverage (R/lib.rs:617-1735, gates.rs). */
NqpuError   nqpu_gate_sx(NqpuState* state, uint32_t qubit);
NqpuError   nqpu_gate_phase(NqpuState* state, uint32_t qubit, double theta);
NqpuError   nqpu_gate_u3(NqpuState* state, uint32_t qubit, double theta, double phi, double lambda);
NqpuError   nqpu_gate_cphase(NqpuState* state, uint32_t control, uint32_t target, double phi);
NqpuError   nqpu_gate_crx(NqpuState* state, uint32_t control, uint32_t target, double theta);
NqpuError   nqpu_gate_cry(NqpuState* state, uint32_t control, uint32_t target, double theta);
NqpuError   nqpu_gate_crz(NqpuState* state, uint32_t control, uint32_t target, double theta);
NqpuError   nqpu_gate_iswap(NqpuState* state, uint32_t q1, uint32_t q2);
NqpuError   nqpu_gate_rzz(NqpuState* state, uint32_t q1, uint32_t q2, double theta);
NqpuError   nqpu_gate_rxx(NqpuState* state, uint32_t q1, uint32_t q2, double theta);
NqpuError   nqpu_gate_ryy(NqpuState* state, uint32_t q1, uint32_t q2, double theta);
NqpuError   nqpu_gate_toffoli(NqpuState* state, uint32_t c1, uint32_t c2, uint32_t target);
NqpuError   nqpu_gate_ccz(NqpuState* state, uint32_t q1, uint32_t q2, uint32_t q3);
NqpuError   nqpu_gate_cswap(NqpuState* state, uint32_t control, uint32_t q1, uint32_t q2);
/* GateType::CU (gates.rs:542): |0><0| x I + e^{i gamma} |1><1| x U3(theta, phi, lambda). */
NqpuError   nqpu_gate_cu(NqpuState* state, uint32_t control, uint32_t target, double theta,
                         double phi, double lambda, double gamma);
/* GateOperations::u2 convention (R/lib.rs:1536): q_lo is bit 0 of the sub-index. */
NqpuError   nqpu_gate_u2(NqpuState* state, uint32_t q_lo, uint32_t q_hi, const NqpuComplex* matrix);
/* R/lib.rs:1705 zero the |1> half of `qubit` and renormalise. */
NqpuError   nqpu_gate_reset_qubit(NqpuState* state, uint32_t qubit);

/* Whole-register reductions (FP64 accumulation). */
/* All <Z_i>, i = 0..n-1, in one pass (len >= n). R/lib.rs:407 for every qubit. */
NqpuError   nqpu_expectation_z_all(const NqpuState* state, double* out, uint32_t len);
/* R/lib.rs:425 / :444 */
NqpuError   nqpu_expectation_x(const NqpuState* state, uint32_t qubit, double* out);
NqpuError   nqpu_expectation_y(const NqpuState* state, uint32_t qubit, double* out);
/* R/lib.rs:465,518 sum_t coeff_t <P_t>; paulis is num_terms strings of n chars
 * 'I','X','Y','Z' (character q acts on qubit q), packed back to back. */
NqpuError   nqpu_expectation_pauli_sum(const NqpuState* state, const char* paulis,
                                       const double* coeffs, uint32_t num_terms, double* out);
/* R/lib.rs:388 |<a|b>|^2 in FP64; the two states may differ in dtype. */
NqpuError   nqpu_fidelity(const NqpuState* a, const NqpuState* b, double* out);
/* Sampling with caller-supplied uniforms in [0,1): out[s] = first i with u[s] < cumsum_i. */
NqpuError   nqpu_sample_with_uniforms(const NqpuState* state, const double* uniforms,
                                      uint32_t num_shots, uint64_t* out);
/* Scale every amplitude by 1/sqrt(norm) (FP64 norm). */
NqpuError   nqpu_state_renormalize(NqpuState* state);

/* Extended circuit builder: every gate of GateType (R/core/gates/gates.rs:8-62). */
NqpuError    nqpu_circuit_add_x(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_y(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_z(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_s(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_t(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_sx(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_ry(NqpuCircuit* c, uint32_t q, double angle);
NqpuError    nqpu_circuit_add_rz(NqpuCircuit* c, uint32_t q, double angle);
NqpuError    nqpu_circuit_add_phase(NqpuCircuit* c, uint32_t q, double angle);
NqpuError    nqpu_circuit_add_u3(NqpuCircuit* c, uint32_t q, double theta, double phi, double lambda);
NqpuError    nqpu_circuit_add_cz(NqpuCircuit* c, uint32_t q1, uint32_t q2);
NqpuError    nqpu_circuit_add_swap(NqpuCircuit* c, uint32_t q1, uint32_t q2);
NqpuError    nqpu_circuit_add_iswap(NqpuCircuit* c, uint32_t q1, uint32_t q2);
NqpuError    nqpu_circuit_add_cphase(NqpuCircuit* c, uint32_t control, uint32_t target, double phi);
NqpuError    nqpu_circuit_add_crx(NqpuCircuit* c, uint32_t control, uint32_t target, double theta);
NqpuError    nqpu_circuit_add_cry(NqpuCircuit* c, uint32_t control, uint32_t target, double theta);
NqpuError    nqpu_circuit_add_crz(NqpuCircuit* c, uint32_t control, uint32_t target, double theta);
NqpuError    nqpu_circuit_add_rzz(NqpuCircuit* c, uint32_t q1, uint32_t q2, double theta);
NqpuError    nqpu_circuit_add_rxx(NqpuCircuit* c, uint32_t q1, uint32_t q2, double theta);
NqpuError    nqpu_circuit_add_ryy(NqpuCircuit* c, uint32_t q1, uint32_t q2, double theta);
NqpuError    nqpu_circuit_add_toffoli(NqpuCircuit* c, uint32_t c1, uint32_t c2, uint32_t target);
NqpuError    nqpu_circuit_add_ccz(NqpuCircuit* c, uint32_t q1, uint32_t q2, uint32_t q3);
NqpuError    nqpu_circuit_add_cswap(NqpuCircuit* c, uint32_t control, uint32_t q1, uint32_t q2);
NqpuError    nqpu_circuit_add_cu(NqpuCircuit* c, uint32_t control, uint32_t target, double theta,
                                 double phi, double lambda, double gamma);
NqpuError    nqpu_circuit_add_custom_1q(NqpuCircuit* c, uint32_t q, const NqpuComplex* matrix);
/* nqpu_gate_custom_2q convention: q1 is the HIGH bit of the sub-index. */
NqpuError    nqpu_circuit_add_custom_2q(NqpuCircuit* c, uint32_t q1, uint32_t q2, const NqpuComplex* matrix);
/* No counterpart in the reference.  All <Z_i> (FP64) of a state that lives in
 * the CALLER's device memory, for callers that cannot allocate device memory:
 * plugins whose host runtime owns the device memory pool, and real-time loops
 * that must not wait on the allocator.  It allocates nothing: the reduction's
 * scratch is a fixed array in this library's device module (about 2.2 MB on
 * every GPU that loads the library, kept until exit).  d_amplitudes: 2^n
 * interleaved (re, im) amplitudes of `dtype`, 16-byte aligned; d_out: n doubles
 * in device memory; cuda_stream: a cudaStream_t (NULL = legacy default
 * stream).  The work is only queued; synchronise the stream before reading
 * d_out.  Limit: complex64 states up to 28 qubits, complex128 up to 27; larger
 * states return NQPU_INVALID_PARAMETER.  The first call on a device (with that
 * device current) resolves the scratch address in the device's primary
 * context and should come before any stream capture; the address is not valid
 * after cudaDeviceReset.  Calls share the scratch, so calls whose kernels
 * overlap on the GPU race. */
NqpuError   nqpu_expectation_z_all_noalloc(const void* d_amplitudes, uint32_t num_qubits,
                                           NqpuDtype dtype, double* d_out, void* cuda_stream);

/* No counterpart in the reference: the bulk form of the nqpu_circuit_add_*
 * calls, for callers that build large circuits or many circuits (one call per
 * circuit instead of one per gate).  Gate i: codes[i] in the gate-code order
 * of nqpu_circuit_get_gate (measure and reset included), qubits[3i..3i+2] and
 * params[4i..4i+3] (slots a gate does not use are ignored), matrices[16i..]
 * row-major for the custom gates only (NULL when there are none; custom 1q
 * reads the first 4 entries).  Each gate is checked as its single add would
 * check it; nothing is appended unless all are valid. */
NqpuError    nqpu_circuit_add_gates(NqpuCircuit* circuit, const uint32_t* codes, const int32_t* qubits,
                                    const double* params, const NqpuComplex* matrices, uint32_t count);
/* Like nqpu_circuit_create with the 34-qubit engine limit. */
NqpuCircuit* nqpu_circuit_create_ex(uint32_t num_qubits);
/* Run with an explicit engine mode. */
NqpuError    nqpu_circuit_execute_ex(const NqpuCircuit* circuit, NqpuState* state, NqpuMode mode);
/* Circuit optimizer pre-pass (CircuitOptimizer, circuits/synthesis/
 * circuit_optimizer.rs:115-735): rewrites the circuit's gate list in place.
 * Levels as the reference's OptimizationLevel: NONE; BASIC = self-inverse
 * cancellation, rotation merging, 1q gate fusion; MODERATE = + commutation;
 * AGGRESSIVE = + peephole patterns.  stats (optional, len values up to 6):
 * original gates, optimized gates, removed, fusions, commutations, cancellations. */
typedef enum { NQPU_OPT_NONE = 0, NQPU_OPT_BASIC = 1, NQPU_OPT_MODERATE = 2, NQPU_OPT_AGGRESSIVE = 3 } NqpuOptLevel;
NqpuError    nqpu_circuit_optimize(NqpuCircuit* circuit, NqpuOptLevel level, uint64_t* stats, uint32_t len);
/* Read gate `index` back: code (the engine's gate-code order, as the Python
 * package's GATE_CODES), qubits[3], params[4], matrix[16] (custom gates). */
NqpuError    nqpu_circuit_get_gate(const NqpuCircuit* circuit, uint32_t index, uint32_t* code, int32_t* qubits,
                                   double* params, NqpuComplex* matrix);

/* Mid-circuit measurement (QuantumSimulator::measure_qubit, lib.rs:1835) and
 * OpenQASM reset: the circuit runs as segments between them; a measurement
 * collapses the state with the next draw of the thread-local RNG (as
 * nqpu_measure); a reset measures the same way and flips the qubit back to |0>
 * when it came out 1 (unlike nqpu_gate_reset_qubit, which keeps the reference's
 * projection, GateOperations::reset_qubit lib.rs:1705).  Batches and the
 * request server take measurement-free circuits. */
NqpuError    nqpu_circuit_add_measure(NqpuCircuit* c, uint32_t q);
NqpuError    nqpu_circuit_add_reset(NqpuCircuit* c, uint32_t q);
/* Execute and return the outcomes of the circuit's measurements in order
 * (*count of them; len must hold every measurement of the circuit). */
NqpuError    nqpu_circuit_execute_measured(const NqpuCircuit* circuit, NqpuState* state, NqpuMode mode,
                                           uint32_t* outcomes, uint32_t len, uint32_t* count);
/* Run the circuit recording a CUDA event between consecutive kernel launches;
 * launch_ms[i] = device time of launch i (i < *count <= len). */
NqpuError    nqpu_circuit_profile(const NqpuCircuit* circuit, NqpuState* state, NqpuMode mode,
                                  float* launch_ms, uint32_t len, uint32_t* count);
/* Tiled-pass kernel configuration per dtype: ctas_per_sm = 1 (one CTA per SM,
 * double-buffered 64 KB tiles), 2 (two CTAs per SM, single-buffered 64 KB
 * tiles) or 4 (four CTAs per SM on 32 KB tiles, one tile qubit fewer).  Plans
 * are built for the configuration in force when a circuit is first run on a
 * state size (a plan built for larger tiles is rebuilt, never run on smaller). */
NqpuError    nqpu_tile_config_set(NqpuDtype dtype, uint32_t ctas_per_sm);
/* Diagnostics (no counterpart in the reference): how many times a tensor-pass
 * engine polls for its MMAs before it gives up (0 = the default, 2^22; at most
 * 2^31 - 1).  never_arrives != 0 points that wait at a barrier nothing
 * arrives on, so it expires: the failure injection of the tests.  On expiry
 * the run returns NQPU_SIMULATION_FAILED; the engine still waits up to 2^24
 * polls for its MMAs in flight before its CTA exits, and the next run starts
 * with a cleared error flag.  Process-wide. */
NqpuError    nqpu_tensor_wait_limit_set(uint32_t polls, int32_t never_arrives);
uint32_t     nqpu_tile_config_get(NqpuDtype dtype);
/* Plan statistics of the last execution of `circuit` in `mode` on an n-qubit state:
 * out[0] = HBM passes (kernel launches over the full state), out[1] = lowered ops,
 * out[2] = register stages (tiled) or fused unitaries (fused, tensor), out[3]
 * (when len >= 4) = bytes of plan tables uploaded host->device per plan build.
 * len >= 3.  For NQPU_MODE_AUTO: the statistics of the modes it picks. */
NqpuError    nqpu_circuit_plan_stats(const NqpuCircuit* circuit, uint32_t num_qubits,
                                     NqpuDtype dtype, NqpuMode mode, uint64_t* out, uint32_t len);
/* The mode NQPU_MODE_AUTO runs the circuit's first gate run (up to its first
 * mid-circuit measurement or reset) in on an n-qubit state of `dtype`:
 * NQPU_MODE_TILED or NQPU_MODE_TENSOR (complex64, n >= 12 only). */
NqpuError    nqpu_circuit_auto_mode(const NqpuCircuit* circuit, uint32_t num_qubits, NqpuDtype dtype,
                                    NqpuMode* out);

/* OpenQASM 2.0 (circuits/formats/qasm.rs:65 parse_qasm, :265 execute_qasm,
 * :363 export): qreg/creg declarations, the qelib1.inc gate set, parameter
 * expressions with pi, measure (terminal: results come from nqpu_sample /
 * nqpu_measure_all), barrier.  NULL on a parse error (unknown gate, undeclared
 * register, bad index, ...); *error_line (optional) gets its 1-based line. */
NqpuCircuit* nqpu_circuit_from_qasm(const char* text, uint32_t* error_line);
/* Qubit count of a circuit (0 on NULL). */
uint32_t     nqpu_circuit_num_qubits(const NqpuCircuit* circuit);
/* OpenQASM 2.0 text of the circuit into out (NUL-terminated, truncated to
 * len-1 bytes); *needed = full length.  NQPU_INVALID_PARAMETER when a gate has
 * no OpenQASM 2.0 form (custom matrices; written as a comment line). */
NqpuError    nqpu_circuit_to_qasm(const NqpuCircuit* circuit, char* out, uint64_t len, uint64_t* needed);

/* ------------------------------------------------------------------ */
/* Batched execution (no counterpart in the reference): many circuits   */
/* of different sizes in one persistent, graph-captured launch; each    */
/* circuit returns <H> of its own 1D Ising Hamiltonian                  */
/* H = sum_i J_i Z_i Z_{i+1} + sum_i h_i X_i (complex64 states).        */
/* ------------------------------------------------------------------ */
typedef struct NqpuBatch NqpuBatch;
typedef enum {
    NQPU_BATCH_SMALL_MAX_QUBITS = 0, /* circuits up to this size run in one CTA's shared memory (5..13) */
    NQPU_BATCH_TILE_QUBITS      = 1, /* tile bits of the larger circuits' passes (10..13) */
    NQPU_BATCH_QUEUE_ORDER      = 2, /* 0: small circuits between pass rounds, 1: first, 2: last */
    NQPU_BATCH_CTAS_PER_SM      = 3, /* persistent CTAs per SM (1..2) */
    /* Polls of a pass tile's bounded dependency wait (>= 1; default 2^26, each
     * poll ~64 ns or more).  When a wait expires, every CTA stops, and
     * nqpu_batch_run returns NQPU_SIMULATION_FAILED; the handle stays usable. */
    NQPU_BATCH_SPIN_LIMIT       = 4,
    /* Failure injection for tests of the bounded waits (0 or 1): 1 leaves the
     * first tile of the first large circuit's first pass out of the queue, so
     * the waits of that circuit's next pass cannot succeed and expire. */
    NQPU_BATCH_DROP_TILE        = 5
} NqpuBatchParam;

NqpuBatch*  nqpu_batch_create(void);
void        nqpu_batch_destroy(NqpuBatch* batch);
/* Append a circuit (5..24 qubits; the gate list is copied) with J[n-1], h[n]. */
NqpuError   nqpu_batch_add_ising(NqpuBatch* batch, const NqpuCircuit* circuit, const double* J,
                                 const double* h, uint32_t* index);
/* No counterpart in the reference: the bulk form of nqpu_batch_add_ising
 * for callers that assemble thousands of circuits (one call instead of two
 * per circuit, gates checked and copied on host threads).  Circuit i has
 * num_qubits[i] (5..24) qubits and the gates gate_offsets[i] ..
 * gate_offsets[i+1]-1 of the flat arrays (the encoding of
 * nqpu_circuit_add_gates: codes, qubits 3 per gate, params 4 per gate,
 * matrices 16 per gate or NULL); J and h hold the circuits' n-1 bonds and n
 * fields one circuit after another.  *first_index = index of circuit 0.
 * Nothing is added unless every circuit is valid. */
NqpuError   nqpu_batch_add_ising_arrays(NqpuBatch* batch, uint32_t count, const uint32_t* num_qubits,
                                        const uint64_t* gate_offsets, const uint32_t* codes,
                                        const int32_t* qubits, const double* params,
                                        const NqpuComplex* matrices, const double* J, const double* h,
                                        uint32_t* first_index);
NqpuError   nqpu_batch_config(NqpuBatch* batch, NqpuBatchParam param, int32_t value);
/* Plan every circuit, upload the task queue and capture the CUDA graph
 * (run() does it on first use). */
NqpuError   nqpu_batch_prepare(NqpuBatch* batch);
/* Replay the graph; results[i] = <H> of circuit i (FP64).  len >= circuits. */
NqpuError   nqpu_batch_run(NqpuBatch* batch, double* results, uint32_t len);
/* out[0..4] = circuits, small circuits, tasks, HBM arena bytes, tiled passes;
 * out[5] (len >= 6) = bytes of tables uploaded host->device by prepare();
 * out[6..9] (len >= 10) = host microseconds of the last prepare() in its
 * phases: plans, table packing, device allocation and upload, graph capture. */
NqpuError   nqpu_batch_stats(const NqpuBatch* batch, uint64_t* out, uint32_t len);
/* Device time of the last run() (CUDA events around the graph replay on the
 * batch's stream: counter resets, the persistent launch, the result copy). */
NqpuError   nqpu_batch_last_run_ms(const NqpuBatch* batch, float* ms);

/* ------------------------------------------------------------------ */
/* Serving (no counterpart in the reference): a request loop that runs  */
/* circuits of mixed sizes on device-resident complex64 states.         */
/* Requests are admitted while others run, as lanes (CUDA streams) and  */
/* HBM budget (2^n x 8 B per state, buddy-allocated in one arena) free  */
/* up, so their kernels overlap on the GPU.  Every handle call is       */
/* thread-safe; results are the same whether a request runs alone or    */
/* in a mix.                                                            */
/* ------------------------------------------------------------------ */
typedef struct NqpuServer NqpuServer;
typedef enum {
    NQPU_REQUEST_ZALL  = 0,  /* all <Z_i> (FP64) */
    NQPU_REQUEST_SHOTS = 1   /* `shots` samples drawn with the request's seed (xorshift64*, as nqpu_set_seed) */
} NqpuRequestKind;
typedef struct {
    uint64_t hbm_budget_bytes; /* resident-state budget; 0 = half of the free device memory */
    uint32_t max_qubits;       /* largest request (<= 32; 0 = 28) */
    uint32_t lanes;            /* requests on the device at once (0 = 16) */
    uint32_t large_lanes;      /* of which large requests may hold (0 = 2) */
    uint32_t large_qubits;     /* "large" = at least this many qubits (0 = 22) */
    uint32_t max_shots;        /* largest shot request (0 = 1024) */
} NqpuServerConfig;

/* NULL on no device, bad config, or a budget below one largest state. */
NqpuServer* nqpu_server_create(const NqpuServerConfig* config);
/* Drops queued requests, waits for running ones, frees everything. */
void        nqpu_server_destroy(NqpuServer* server);
/* Plans the circuit (copied; the handle may be destroyed afterwards) and
 * queues it; *request_id > 0. */
NqpuError   nqpu_server_submit(NqpuServer* server, const NqpuCircuit* circuit, NqpuRequestKind kind,
                               uint32_t shots, uint64_t seed, uint64_t* request_id);
/* *done = 1 once the request finished (non-blocking). */
NqpuError   nqpu_server_poll(NqpuServer* server, uint64_t request_id, int32_t* done);
/* Block until the request (request_id = 0: every submitted request) finished;
 * NQPU_SIMULATION_FAILED after timeout_s (<= 0: one hour). */
NqpuError   nqpu_server_wait(NqpuServer* server, uint64_t request_id, double timeout_s);
/* Copy a finished request's result and release it: out_z[0..n) for ZALL,
 * out_shots[0..shots) for SHOTS; timing_ms (optional, 3 values) = queued,
 * running, total milliseconds from submit to completion. */
NqpuError   nqpu_server_result(NqpuServer* server, uint64_t request_id, double* out_z, uint32_t z_len,
                               uint64_t* out_shots, uint32_t shots_len, double* timing_ms);
/* Withdraw a request that is still queued (not yet admitted to a lane): it
 * never runs and its id is forgotten (later calls with it return
 * NQPU_INVALID_HANDLE).  NQPU_INVALID_PARAMETER when the request is already
 * running or finished (it completes normally); NQPU_INVALID_HANDLE for an
 * unknown id. */
NqpuError   nqpu_server_cancel(NqpuServer* server, uint64_t request_id);
/* out[0..7] = submitted, completed, failed, running, queued, peak resident
 * bytes, arena bytes, peak concurrent requests; out[8] (len >= 9) = cancelled
 * requests.  len >= 8. */
NqpuError   nqpu_server_stats(NqpuServer* server, uint64_t* out, uint32_t len);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* NQPU_B200_H */
