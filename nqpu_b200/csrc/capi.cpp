// C ABI of the engine (include/nqpu_b200.h).
//
// Every entry point keeps the reference C FFI's argument checks and error codes
// (sdk/rust/src/infra/bindings/c_ffi.rs:789-1470): NULL handle ->
// NQPU_NULL_POINTER, qubit >= n -> NQPU_INVALID_QUBIT, non-finite angle or equal
// qubits -> NQPU_INVALID_PARAMETER.  CUDA failures map to
// NQPU_SIMULATION_FAILED and device OOM to NQPU_ALLOCATION_FAILED.  The
// computation itself always runs on the GPU: there is no host fallback.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/nqpu_b200.h"
#include "engine.h"
#include "kernels.h"
#include "planner.h"

using namespace nqpu;

// ---------------------------------------------------------------------------
// Thread-local xorshift64* RNG (same generator, seeding and [0,1) mapping as
// c_ffi.rs:49-66 / :1444), so seeded measurement and sampling draw the same
// uniforms as the reference C FFI.
// ---------------------------------------------------------------------------
static thread_local uint64_t t_rng_state = 0x853c49e6748fea9bull;

double nqpu::next_random_f64() {
  uint64_t s = t_rng_state;
  s ^= s >> 12;
  s ^= s << 25;
  s ^= s >> 27;
  t_rng_state = s;
  const uint64_t v = s * 0x2545F4914F6CDD1Dull;
  return double(v >> 11) / double(1ull << 53);
}

extern "C" void nqpu_set_seed(uint64_t seed) {
  t_rng_state = seed == 0 ? 0x853c49e6748fea9bull : seed;
}

extern "C" void nqpu_set_num_threads(uint32_t) {}

// ---------------------------------------------------------------------------
// Handles
// ---------------------------------------------------------------------------
static bool is_finite_param(double x) { return std::isfinite(x); }

static NqpuError map_cuda(cudaError_t e) {
  if (e == cudaSuccess) return NQPU_OK;
  if (e == cudaErrorMemoryAllocation) return NQPU_ALLOCATION_FAILED;
  return NQPU_SIMULATION_FAILED;
}

#define NQ_TRY(expr)                                  \
  do {                                                \
    cudaError_t _e = (expr);                          \
    if (_e != cudaSuccess) return map_cuda(_e);       \
  } while (0)

static NqpuState* as_handle(StateImpl* s) { return reinterpret_cast<NqpuState*>(s); }
static StateImpl* S(NqpuState* h) { return reinterpret_cast<StateImpl*>(h); }
static const StateImpl* S(const NqpuState* h) { return reinterpret_cast<const StateImpl*>(h); }
static CircuitImpl* Cc(NqpuCircuit* h) { return reinterpret_cast<CircuitImpl*>(h); }
static const CircuitImpl* Cc(const NqpuCircuit* h) { return reinterpret_cast<const CircuitImpl*>(h); }

// ---------------------------------------------------------------------------
// State management
// ---------------------------------------------------------------------------
extern "C" NqpuState* nqpu_state_create_ex(uint32_t num_qubits, NqpuDtype dtype) {
  if (num_qubits == 0 || num_qubits > uint32_t(kMaxQubits)) return nullptr;
  if (dtype != NQPU_C128 && dtype != NQPU_C64) return nullptr;
  StateImpl* s = state_new(num_qubits, dtype == NQPU_C64 ? DType::C64 : DType::C128);
  return s ? as_handle(s) : nullptr;
}

extern "C" NqpuState* nqpu_state_create(uint32_t num_qubits) {
  if (num_qubits == 0 || num_qubits > 30) return nullptr;  // c_ffi.rs:790
  return nqpu_state_create_ex(num_qubits, NQPU_C128);
}

extern "C" void nqpu_state_destroy(NqpuState* state) {
  if (state) state_free(S(state));
}

extern "C" NqpuState* nqpu_state_clone(const NqpuState* state) {
  if (!state) return nullptr;
  const StateImpl* src = S(state);
  StateImpl* dst = state_new(src->n, src->dt);
  if (!dst) return nullptr;
  if (cudaStreamSynchronize(src->stream) != cudaSuccess ||
      cudaMemcpyAsync(dst->amp, src->amp, src->bytes, cudaMemcpyDeviceToDevice, dst->stream) != cudaSuccess ||
      cudaStreamSynchronize(dst->stream) != cudaSuccess) {
    state_free(dst);
    return nullptr;
  }
  return as_handle(dst);
}

extern "C" uint32_t nqpu_state_num_qubits(const NqpuState* state) {
  return state ? S(state)->n : 0;
}

extern "C" NqpuDtype nqpu_state_dtype(const NqpuState* state) {
  return (state && S(state)->dt == DType::C64) ? NQPU_C64 : NQPU_C128;
}

extern "C" void* nqpu_state_cuda_stream(const NqpuState* state) {
  return state ? static_cast<void*>(S(state)->stream) : nullptr;
}

extern "C" NqpuError nqpu_state_synchronize(const NqpuState* state) {
  if (!state) return NQPU_NULL_POINTER;
  NQ_TRY(cudaStreamSynchronize(S(state)->stream));
  return NQPU_OK;
}

extern "C" NqpuError nqpu_state_get_amplitude(const NqpuState* state, uint64_t index, NqpuComplex* out) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  if (index >= (1ull << s->n)) return NQPU_INVALID_PARAMETER;
  const size_t ab = amp_bytes(s->dt);
  NQ_TRY(cudaMemcpyAsync(s->h_small, static_cast<const char*>(s->amp) + index * ab, ab,
                         cudaMemcpyDeviceToHost, s->stream));
  NQ_TRY(cudaStreamSynchronize(s->stream));
  if (s->dt == DType::C64) {
    const float* f = reinterpret_cast<const float*>(s->h_small);
    out->re = f[0];
    out->im = f[1];
  } else {
    out->re = s->h_small[0];
    out->im = s->h_small[1];
  }
  return NQPU_OK;
}

extern "C" NqpuError nqpu_state_set_amplitude(NqpuState* state, uint64_t index, NqpuComplex amp) {
  if (!state) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  if (index >= (1ull << s->n)) return NQPU_INVALID_PARAMETER;
  const size_t ab = amp_bytes(s->dt);
  NQ_TRY(cudaStreamSynchronize(s->stream));
  if (s->dt == DType::C64) {
    float* f = reinterpret_cast<float*>(s->h_small);
    f[0] = float(amp.re);
    f[1] = float(amp.im);
  } else {
    s->h_small[0] = amp.re;
    s->h_small[1] = amp.im;
  }
  NQ_TRY(cudaMemcpyAsync(static_cast<char*>(s->amp) + index * ab, s->h_small, ab,
                         cudaMemcpyHostToDevice, s->stream));
  NQ_TRY(cudaStreamSynchronize(s->stream));
  return NQPU_OK;
}

extern "C" NqpuError nqpu_state_get_amplitudes(const NqpuState* state, NqpuComplex* out, uint64_t len) {
  if (!state || !out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  const uint64_t dim = 1ull << s->n;
  if (len < dim) return NQPU_INVALID_PARAMETER;
  return map_cuda(state_download_c128(s, out));
}

extern "C" NqpuError nqpu_state_set_amplitudes(NqpuState* state, const NqpuComplex* in, uint64_t len) {
  if (!state || !in) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  const uint64_t dim = 1ull << s->n;
  if (len < dim) return NQPU_INVALID_PARAMETER;
  return map_cuda(state_upload_c128(s, in));
}

extern "C" NqpuError nqpu_state_probabilities(const NqpuState* state, double* out, uint64_t len) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  if (len < (1ull << s->n)) return NQPU_INVALID_PARAMETER;
  return map_cuda(state_probabilities(s, out));
}

extern "C" double nqpu_state_norm(const NqpuState* state) {
  if (!state) return -1.0;
  double tot = 0.0;
  if (state_zsums(S(state), nullptr, &tot) != cudaSuccess) return -1.0;
  return tot;
}

extern "C" NqpuError nqpu_state_reset(NqpuState* state) {
  if (!state) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  NQ_TRY(launch_set_basis(s->dt, s->amp, int(s->n), 0, s->stream, device_sms()));
  return NQPU_OK;
}

extern "C" NqpuError nqpu_state_set_basis(NqpuState* state, uint64_t index) {
  if (!state) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  if (index >= (1ull << s->n)) return NQPU_INVALID_PARAMETER;
  NQ_TRY(launch_set_basis(s->dt, s->amp, int(s->n), index, s->stream, device_sms()));
  return NQPU_OK;
}

extern "C" NqpuError nqpu_state_renormalize(NqpuState* state) {
  if (!state) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  double tot = 0.0;
  NQ_TRY(state_zsums(s, nullptr, &tot));
  if (!(tot > 0.0)) return NQPU_SIMULATION_FAILED;
  NQ_TRY(launch_scale(s->dt, s->amp, int(s->n), 1.0 / std::sqrt(tot), s->stream, device_sms()));
  return NQPU_OK;
}

// ---------------------------------------------------------------------------
// Gates (one per-gate kernel launch each, stream-ordered)
// ---------------------------------------------------------------------------
static NqpuError apply_rec(NqpuState* state, const GateRec& g) {
  if (!state) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  const int ar = gate_arity(g.code);
  for (int i = 0; i < ar; ++i)
    if (g.q[i] < 0 || uint32_t(g.q[i]) >= s->n) return NQPU_INVALID_QUBIT;
  for (int i = 0; i < ar; ++i)
    for (int j = i + 1; j < ar; ++j)
      if (g.q[i] == g.q[j]) return NQPU_INVALID_PARAMETER;
  for (int i = 0; i < 4; ++i)
    if (!is_finite_param(g.p[i])) return NQPU_INVALID_PARAMETER;
  const Op op = lower_gate(g);
  NQ_TRY(launch_pergate(s->dt, s->amp, int(s->n), op, s->stream, device_sms()));
  return NQPU_OK;
}

static GateRec mk(uint8_t code, int a, int b = 0, int c = 0, double p0 = 0, double p1 = 0,
                  double p2 = 0, double p3 = 0) {
  GateRec g;
  g.code = code;
  g.nq = uint8_t(gate_arity(code));
  g.q[0] = a; g.q[1] = b; g.q[2] = c;
  g.p[0] = p0; g.p[1] = p1; g.p[2] = p2; g.p[3] = p3;
  return g;
}

// qubit arguments arrive as uint32; anything >= 2^31 is out of range anyway
static int qi(uint32_t q) { return q > 0x7fffffffu ? 0x7fffffff : int(q); }

#define NQ_GATE1(NAME, CODE) \
  extern "C" NqpuError NAME(NqpuState* state, uint32_t q) { return apply_rec(state, mk(CODE, qi(q))); }
#define NQ_GATE1P(NAME, CODE)                                          \
  extern "C" NqpuError NAME(NqpuState* state, uint32_t q, double a) { \
    return apply_rec(state, mk(CODE, qi(q), 0, 0, a));                 \
  }
#define NQ_GATE2(NAME, CODE)                                                 \
  extern "C" NqpuError NAME(NqpuState* state, uint32_t a, uint32_t b) {      \
    return apply_rec(state, mk(CODE, qi(a), qi(b)));                         \
  }
#define NQ_GATE2P(NAME, CODE)                                                      \
  extern "C" NqpuError NAME(NqpuState* state, uint32_t a, uint32_t b, double t) { \
    return apply_rec(state, mk(CODE, qi(a), qi(b), 0, t));                         \
  }
#define NQ_GATE3(NAME, CODE)                                                        \
  extern "C" NqpuError NAME(NqpuState* state, uint32_t a, uint32_t b, uint32_t c) { \
    return apply_rec(state, mk(CODE, qi(a), qi(b), qi(c)));                         \
  }

NQ_GATE1(nqpu_gate_h, G_H)
NQ_GATE1(nqpu_gate_x, G_X)
NQ_GATE1(nqpu_gate_y, G_Y)
NQ_GATE1(nqpu_gate_z, G_Z)
NQ_GATE1(nqpu_gate_s, G_S)
NQ_GATE1(nqpu_gate_t, G_T)
NQ_GATE1(nqpu_gate_sx, G_SX)
NQ_GATE1P(nqpu_gate_rx, G_RX)
NQ_GATE1P(nqpu_gate_ry, G_RY)
NQ_GATE1P(nqpu_gate_rz, G_RZ)
NQ_GATE1P(nqpu_gate_phase, G_P)
NQ_GATE2(nqpu_gate_cx, G_CX)
NQ_GATE2(nqpu_gate_cz, G_CZ)
NQ_GATE2(nqpu_gate_swap, G_SWAP)
NQ_GATE2(nqpu_gate_iswap, G_ISWAP)
NQ_GATE2P(nqpu_gate_cphase, G_CP)
NQ_GATE2P(nqpu_gate_crx, G_CRX)
NQ_GATE2P(nqpu_gate_cry, G_CRY)
NQ_GATE2P(nqpu_gate_crz, G_CRZ)
NQ_GATE2P(nqpu_gate_rzz, G_RZZ)
NQ_GATE2P(nqpu_gate_rxx, G_RXX)
NQ_GATE2P(nqpu_gate_ryy, G_RYY)
NQ_GATE3(nqpu_gate_toffoli, G_CCX)
NQ_GATE3(nqpu_gate_ccz, G_CCZ)
NQ_GATE3(nqpu_gate_cswap, G_CSWAP)

extern "C" NqpuError nqpu_gate_u3(NqpuState* state, uint32_t q, double th, double ph, double la) {
  return apply_rec(state, mk(G_U3, qi(q), 0, 0, th, ph, la));
}

extern "C" NqpuError nqpu_gate_cu(NqpuState* state, uint32_t c, uint32_t t, double th, double ph,
                                   double la, double ga) {
  return apply_rec(state, mk(G_CU, qi(c), qi(t), 0, th, ph, la, ga));
}

extern "C" NqpuError nqpu_gate_custom_1q(NqpuState* state, uint32_t qubit, const NqpuComplex* matrix) {
  if (!state) return NQPU_NULL_POINTER;
  if (!matrix) return NQPU_NULL_POINTER;
  GateRec g = mk(G_CUSTOM1, qi(qubit));
  for (int i = 0; i < 4; ++i) g.m[i] = cplx(matrix[i].re, matrix[i].im);
  return apply_rec(state, g);
}

extern "C" NqpuError nqpu_gate_custom_2q(NqpuState* state, uint32_t q1, uint32_t q2, const NqpuComplex* matrix) {
  if (!state) return NQPU_NULL_POINTER;
  if (!matrix) return NQPU_NULL_POINTER;
  GateRec g = mk(G_CUSTOM2_FFI, qi(q1), qi(q2));
  for (int i = 0; i < 16; ++i) g.m[i] = cplx(matrix[i].re, matrix[i].im);
  return apply_rec(state, g);
}

extern "C" NqpuError nqpu_gate_u2(NqpuState* state, uint32_t q_lo, uint32_t q_hi, const NqpuComplex* matrix) {
  if (!state) return NQPU_NULL_POINTER;
  if (!matrix) return NQPU_NULL_POINTER;
  GateRec g = mk(G_U2_LO, qi(q_lo), qi(q_hi));
  for (int i = 0; i < 16; ++i) g.m[i] = cplx(matrix[i].re, matrix[i].im);
  return apply_rec(state, g);
}

extern "C" NqpuError nqpu_gate_reset_qubit(NqpuState* state, uint32_t qubit) {
  if (!state) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  if (qubit >= s->n) return NQPU_INVALID_QUBIT;
  NQ_TRY(state_reset_qubit(s, qubit));
  return NQPU_OK;
}

// ---------------------------------------------------------------------------
// Measurement and reductions
// ---------------------------------------------------------------------------
static NqpuError measure_one(StateImpl* s, uint32_t qubit, NqpuMeasurement* out) {
  uint32_t outcome = 0;
  double po = 0.0;
  NQ_TRY(state_measure(s, qubit, &outcome, &po));
  out->outcome = outcome;
  out->probability = po;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_measure(NqpuState* state, uint32_t qubit, NqpuMeasurement* out) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  if (qubit >= s->n) return NQPU_INVALID_QUBIT;
  return measure_one(s, qubit, out);
}

extern "C" NqpuError nqpu_measure_all(NqpuState* state, uint32_t* out, uint32_t num_qubits) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  StateImpl* s = S(state);
  if (num_qubits != s->n) return NQPU_INVALID_PARAMETER;
  for (uint32_t q = 0; q < s->n; ++q) {
    NqpuMeasurement m;
    NqpuError e = measure_one(s, q, &m);
    if (e != NQPU_OK) return e;
    out[q] = m.outcome;
  }
  return NQPU_OK;
}

extern "C" NqpuError nqpu_expectation_z(const NqpuState* state, uint32_t qubit, double* out) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  if (qubit >= s->n) return NQPU_INVALID_QUBIT;
  std::vector<double> z(s->n + 1);
  NQ_TRY(state_zsums(s, z.data(), nullptr));
  *out = z[0] - 2.0 * z[1 + qubit];
  return NQPU_OK;
}

extern "C" NqpuError nqpu_expectation_z_all(const NqpuState* state, double* out, uint32_t len) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  if (len < s->n) return NQPU_INVALID_PARAMETER;
  std::vector<double> z(s->n + 1);
  NQ_TRY(state_zsums(s, z.data(), nullptr));
  for (uint32_t q = 0; q < s->n; ++q) out[q] = z[0] - 2.0 * z[1 + q];
  return NQPU_OK;
}

static NqpuError pauli_expect(const StateImpl* s, uint64_t xm, uint64_t zm, uint64_t ym, double* out) {
  double r[2];
  NQ_TRY(state_pauli(s, xm, zm, ym, r));
  *out = r[0];
  return NQPU_OK;
}

extern "C" NqpuError nqpu_expectation_x(const NqpuState* state, uint32_t qubit, double* out) {
  if (!state || !out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  if (qubit >= s->n) return NQPU_INVALID_QUBIT;
  return pauli_expect(s, 1ull << qubit, 0, 0, out);
}

extern "C" NqpuError nqpu_expectation_y(const NqpuState* state, uint32_t qubit, double* out) {
  if (!state || !out) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  if (qubit >= s->n) return NQPU_INVALID_QUBIT;
  return pauli_expect(s, 1ull << qubit, 1ull << qubit, 1ull << qubit, out);
}

extern "C" NqpuError nqpu_expectation_pauli_sum(const NqpuState* state, const char* paulis,
                                                const double* coeffs, uint32_t num_terms, double* out) {
  if (!state || !out) return NQPU_NULL_POINTER;
  if (num_terms > 0 && (!paulis || !coeffs)) return NQPU_NULL_POINTER;
  const StateImpl* s = S(state);
  const uint32_t n = s->n;
  // Parse all terms first (invalid characters -> InvalidParameter, nothing runs).
  std::vector<std::tuple<uint64_t, uint64_t, uint64_t>> masks(num_terms);
  for (uint32_t t = 0; t < num_terms; ++t) {
    uint64_t xm = 0, zm = 0, ym = 0;
    for (uint32_t q = 0; q < n; ++q) {
      const char ch = paulis[size_t(t) * n + q];
      switch (ch) {
        case 'I': break;
        case 'X': xm |= 1ull << q; break;
        case 'Y': xm |= 1ull << q; zm |= 1ull << q; ym |= 1ull << q; break;
        case 'Z': zm |= 1ull << q; break;
        default: return NQPU_INVALID_PARAMETER;
      }
    }
    if (!is_finite_param(coeffs[t])) return NQPU_INVALID_PARAMETER;
    masks[t] = std::make_tuple(xm, zm, ym);
  }
  double total = 0.0;
  for (uint32_t t = 0; t < num_terms; ++t) {
    double v = 0.0;
    NqpuError e = pauli_expect(s, std::get<0>(masks[t]), std::get<1>(masks[t]), std::get<2>(masks[t]), &v);
    if (e != NQPU_OK) return e;
    total += coeffs[t] * v;
  }
  *out = total;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_fidelity(const NqpuState* a, const NqpuState* b, double* out) {
  if (!a || !b || !out) return NQPU_NULL_POINTER;
  const StateImpl* sa = S(a);
  const StateImpl* sb = S(b);
  if (sa->n != sb->n) {  // R/lib.rs:389 dims differ -> 0.0
    *out = 0.0;
    return NQPU_OK;
  }
  double r[2];
  NQ_TRY(state_inner(sa, sb, r));
  *out = r[0] * r[0] + r[1] * r[1];
  return NQPU_OK;
}

extern "C" NqpuError nqpu_sample_with_uniforms(const NqpuState* state, const double* uniforms,
                                               uint32_t num_shots, uint64_t* out) {
  if (!state || !out) return NQPU_NULL_POINTER;
  if (num_shots == 0) return NQPU_OK;
  if (!uniforms) return NQPU_NULL_POINTER;
  return map_cuda(state_sample(S(state), uniforms, num_shots, out));
}

extern "C" NqpuError nqpu_sample(const NqpuState* state, uint32_t num_shots, uint64_t* out) {
  if (!state) return NQPU_NULL_POINTER;
  if (!out) return NQPU_NULL_POINTER;
  if (num_shots == 0) return NQPU_OK;
  std::vector<double> u(num_shots);
  for (auto& x : u) x = next_random_f64();  // c_ffi.rs:608 draws one r per shot
  return map_cuda(state_sample(S(state), u.data(), num_shots, out));
}

// ---------------------------------------------------------------------------
// Circuits
// ---------------------------------------------------------------------------
extern "C" NqpuCircuit* nqpu_circuit_create_ex(uint32_t num_qubits) {
  if (num_qubits == 0 || num_qubits > uint32_t(kMaxQubits)) return nullptr;
  auto* c = new (std::nothrow) CircuitImpl();
  if (!c) return nullptr;
  c->n = num_qubits;
  return reinterpret_cast<NqpuCircuit*>(c);
}

extern "C" NqpuCircuit* nqpu_circuit_create(uint32_t num_qubits) {
  if (num_qubits == 0 || num_qubits > 30) return nullptr;  // c_ffi.rs:1260
  return nqpu_circuit_create_ex(num_qubits);
}

extern "C" void nqpu_circuit_destroy(NqpuCircuit* circuit) {
  if (circuit) circuit_free(Cc(circuit));
}

static NqpuError check_rec(const CircuitImpl* c, const GateRec& g) {
  const int ar = gate_arity(g.code);
  for (int i = 0; i < ar; ++i)
    if (g.q[i] < 0 || uint32_t(g.q[i]) >= c->n) return NQPU_INVALID_QUBIT;
  for (int i = 0; i < ar; ++i)
    for (int j = i + 1; j < ar; ++j)
      if (g.q[i] == g.q[j]) return NQPU_INVALID_PARAMETER;
  for (int i = 0; i < 4; ++i)
    if (!is_finite_param(g.p[i])) return NQPU_INVALID_PARAMETER;
  return NQPU_OK;
}

static NqpuError add_rec(NqpuCircuit* circuit, const GateRec& g) {
  if (!circuit) return NQPU_NULL_POINTER;
  CircuitImpl* c = Cc(circuit);
  const NqpuError e = check_rec(c, g);
  if (e != NQPU_OK) return e;
  c->gates.push_back(g);
  c->version++;
  return NQPU_OK;
}

#define NQ_CADD1(NAME, CODE) \
  extern "C" NqpuError NAME(NqpuCircuit* c, uint32_t q) { return add_rec(c, mk(CODE, qi(q))); }
#define NQ_CADD1P(NAME, CODE)                                            \
  extern "C" NqpuError NAME(NqpuCircuit* c, uint32_t q, double a) {     \
    return add_rec(c, mk(CODE, qi(q), 0, 0, a));                         \
  }
#define NQ_CADD2(NAME, CODE)                                             \
  extern "C" NqpuError NAME(NqpuCircuit* c, uint32_t a, uint32_t b) {   \
    return add_rec(c, mk(CODE, qi(a), qi(b)));                           \
  }
#define NQ_CADD2P(NAME, CODE)                                                    \
  extern "C" NqpuError NAME(NqpuCircuit* c, uint32_t a, uint32_t b, double t) { \
    return add_rec(c, mk(CODE, qi(a), qi(b), 0, t));                             \
  }
#define NQ_CADD3(NAME, CODE)                                                       \
  extern "C" NqpuError NAME(NqpuCircuit* c, uint32_t a, uint32_t b, uint32_t d) { \
    return add_rec(c, mk(CODE, qi(a), qi(b), qi(d)));                              \
  }

NQ_CADD1(nqpu_circuit_add_h, G_H)
NQ_CADD1(nqpu_circuit_add_x, G_X)
NQ_CADD1(nqpu_circuit_add_y, G_Y)
NQ_CADD1(nqpu_circuit_add_z, G_Z)
NQ_CADD1(nqpu_circuit_add_s, G_S)
NQ_CADD1(nqpu_circuit_add_t, G_T)
NQ_CADD1(nqpu_circuit_add_measure, G_MEASURE)
NQ_CADD1(nqpu_circuit_add_reset, G_RESET)
NQ_CADD1(nqpu_circuit_add_sx, G_SX)
NQ_CADD1P(nqpu_circuit_add_rx, G_RX)
NQ_CADD1P(nqpu_circuit_add_ry, G_RY)
NQ_CADD1P(nqpu_circuit_add_rz, G_RZ)
NQ_CADD1P(nqpu_circuit_add_phase, G_P)
NQ_CADD2(nqpu_circuit_add_cx, G_CX)
NQ_CADD2(nqpu_circuit_add_cz, G_CZ)
NQ_CADD2(nqpu_circuit_add_swap, G_SWAP)
NQ_CADD2(nqpu_circuit_add_iswap, G_ISWAP)
NQ_CADD2P(nqpu_circuit_add_cphase, G_CP)
NQ_CADD2P(nqpu_circuit_add_crx, G_CRX)
NQ_CADD2P(nqpu_circuit_add_cry, G_CRY)
NQ_CADD2P(nqpu_circuit_add_crz, G_CRZ)
NQ_CADD2P(nqpu_circuit_add_rzz, G_RZZ)
NQ_CADD2P(nqpu_circuit_add_rxx, G_RXX)
NQ_CADD2P(nqpu_circuit_add_ryy, G_RYY)
NQ_CADD3(nqpu_circuit_add_toffoli, G_CCX)
NQ_CADD3(nqpu_circuit_add_ccz, G_CCZ)
NQ_CADD3(nqpu_circuit_add_cswap, G_CSWAP)

extern "C" NqpuError nqpu_circuit_add_u3(NqpuCircuit* c, uint32_t q, double th, double ph, double la) {
  return add_rec(c, mk(G_U3, qi(q), 0, 0, th, ph, la));
}

extern "C" NqpuError nqpu_circuit_add_cu(NqpuCircuit* c, uint32_t ctl, uint32_t t, double th,
                                         double ph, double la, double ga) {
  return add_rec(c, mk(G_CU, qi(ctl), qi(t), 0, th, ph, la, ga));
}

extern "C" NqpuError nqpu_circuit_add_custom_1q(NqpuCircuit* c, uint32_t q, const NqpuComplex* matrix) {
  if (!c || !matrix) return NQPU_NULL_POINTER;
  GateRec g = mk(G_CUSTOM1, qi(q));
  for (int i = 0; i < 4; ++i) g.m[i] = cplx(matrix[i].re, matrix[i].im);
  return add_rec(c, g);
}

extern "C" NqpuError nqpu_circuit_add_custom_2q(NqpuCircuit* c, uint32_t q1, uint32_t q2, const NqpuComplex* matrix) {
  if (!c || !matrix) return NQPU_NULL_POINTER;
  GateRec g = mk(G_CUSTOM2_FFI, qi(q1), qi(q2));
  for (int i = 0; i < 16; ++i) g.m[i] = cplx(matrix[i].re, matrix[i].im);
  return add_rec(c, g);
}

NqpuError nqpu::circuit_append_gates(CircuitImpl* c, const uint32_t* codes, const int32_t* qubits,
                                     const double* params, const NqpuComplex* matrices, size_t count) {
  if (count == 0) return NQPU_OK;
  if (!codes || !qubits || !params) return NQPU_NULL_POINTER;
  // the records are written in place after the existing gates and dropped
  // again when any of them is rejected (the circuit is then unchanged)
  const size_t base = c->gates.size();
  try {
    c->gates.resize(base + size_t(count));
  } catch (...) {
    return NQPU_ALLOCATION_FAILED;
  }
  // index arithmetic in size_t: 16 * count overflows 32 bits above 2^28 gates
  for (size_t i = 0; i < size_t(count); ++i) {
    NqpuError e = NQPU_OK;
    GateRec& g = c->gates[base + i];
    if (codes[i] >= uint32_t(G_COUNT)) {
      e = NQPU_INVALID_PARAMETER;
    } else {
      g.code = uint8_t(codes[i]);
      g.nq = uint8_t(gate_arity(g.code));
      for (int k = 0; k < 3; ++k) g.q[k] = k < g.nq ? qubits[3 * i + size_t(k)] : 0;  // unused slots ignored
      for (int k = 0; k < 4; ++k) g.p[k] = params[4 * i + size_t(k)];
      if (g.code == G_CUSTOM1 || g.code == G_CUSTOM2_FFI || g.code == G_U2_LO) {
        if (!matrices) {
          e = NQPU_NULL_POINTER;
        } else {
          const int nm = g.code == G_CUSTOM1 ? 4 : 16;
          for (int k = 0; k < nm; ++k)
            g.m[k] = cplx(matrices[16 * i + size_t(k)].re, matrices[16 * i + size_t(k)].im);
        }
      }
      if (e == NQPU_OK) e = check_rec(c, g);
    }
    if (e != NQPU_OK) {
      c->gates.resize(base);
      return e;
    }
  }
  c->version++;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_circuit_add_gates(NqpuCircuit* circuit, const uint32_t* codes, const int32_t* qubits,
                                            const double* params, const NqpuComplex* matrices, uint32_t count) {
  if (!circuit) return NQPU_NULL_POINTER;
  return circuit_append_gates(Cc(circuit), codes, qubits, params, matrices, size_t(count));
}

static bool mode_ok(NqpuMode mode) {
  return mode == NQPU_MODE_TILED || mode == NQPU_MODE_PERGATE || mode == NQPU_MODE_FUSED || mode == NQPU_MODE_TENSOR ||
         mode == NQPU_MODE_AUTO;
}

extern "C" NqpuError nqpu_circuit_execute_ex(const NqpuCircuit* circuit, NqpuState* state, NqpuMode mode) {
  if (!circuit) return NQPU_NULL_POINTER;
  if (!state) return NQPU_NULL_POINTER;
  const CircuitImpl* c = Cc(circuit);
  StateImpl* s = S(state);
  if (c->n > s->n) return NQPU_INVALID_PARAMETER;  // c_ffi.rs:1360
  if (!mode_ok(mode)) return NQPU_INVALID_PARAMETER;
  // the fused and tensor modes run complex64 states of >= 12 qubits (5 fused + 7 row bits)
  if ((mode == NQPU_MODE_FUSED || mode == NQPU_MODE_TENSOR) && (s->dt != DType::C64 || s->n < 12))
    return NQPU_INVALID_PARAMETER;
  cudaError_t e = circuit_run(const_cast<CircuitImpl*>(c), s, int(mode));
  if (e != cudaSuccess) return map_cuda(e);
  NQ_TRY(cudaStreamSynchronize(s->stream));
  return NQPU_OK;
}

extern "C" NqpuError nqpu_circuit_execute_measured(const NqpuCircuit* circuit, NqpuState* state, NqpuMode mode,
                                                   uint32_t* outcomes, uint32_t len, uint32_t* count) {
  if (!circuit || !state || !count) return NQPU_NULL_POINTER;
  const CircuitImpl* c = Cc(circuit);
  StateImpl* s = S(state);
  if (c->n > s->n) return NQPU_INVALID_PARAMETER;
  if (!mode_ok(mode)) return NQPU_INVALID_PARAMETER;
  if ((mode == NQPU_MODE_FUSED || mode == NQPU_MODE_TENSOR) && (s->dt != DType::C64 || s->n < 12))
    return NQPU_INVALID_PARAMETER;
  uint32_t nmeas = 0;
  for (const GateRec& g : c->gates) nmeas += g.code == G_MEASURE ? 1u : 0u;
  if (nmeas > 0 && (!outcomes || len < nmeas)) return NQPU_INVALID_PARAMETER;
  std::vector<uint32_t> out;
  cudaError_t e = circuit_run(const_cast<CircuitImpl*>(c), s, int(mode), nullptr, &out);
  if (e != cudaSuccess) return map_cuda(e);
  NQ_TRY(cudaStreamSynchronize(s->stream));
  for (size_t i = 0; i < out.size(); ++i) outcomes[i] = out[i];
  *count = uint32_t(out.size());
  return NQPU_OK;
}

extern "C" NqpuError nqpu_circuit_profile(const NqpuCircuit* circuit, NqpuState* state, NqpuMode mode,
                                          float* launch_ms, uint32_t len, uint32_t* count) {
  if (!circuit || !state || !launch_ms || !count) return NQPU_NULL_POINTER;
  const CircuitImpl* c = Cc(circuit);
  StateImpl* s = S(state);
  if (c->n > s->n) return NQPU_INVALID_PARAMETER;
  if (!mode_ok(mode)) return NQPU_INVALID_PARAMETER;
  if ((mode == NQPU_MODE_FUSED || mode == NQPU_MODE_TENSOR) && (s->dt != DType::C64 || s->n < 12))
    return NQPU_INVALID_PARAMETER;
  std::vector<cudaEvent_t> ev;
  cudaError_t e = circuit_run(const_cast<CircuitImpl*>(c), s, int(mode), &ev);
  cudaError_t e2 = cudaStreamSynchronize(s->stream);
  uint32_t k = 0;
  for (size_t i = 0; i + 1 < ev.size() && k < len; ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
    launch_ms[k++] = ms;
  }
  for (auto x : ev) cudaEventDestroy(x);
  *count = k;
  if (e != cudaSuccess) return map_cuda(e);
  if (e2 != cudaSuccess) return map_cuda(e2);
  return NQPU_OK;
}

extern "C" NqpuError nqpu_circuit_execute(const NqpuCircuit* circuit, NqpuState* state) {
  return nqpu_circuit_execute_ex(circuit, state, NQPU_MODE_TILED);
}

extern "C" uint32_t nqpu_circuit_gate_count(const NqpuCircuit* circuit) {
  return circuit ? uint32_t(Cc(circuit)->gates.size()) : 0;
}

extern "C" uint32_t nqpu_circuit_depth(const NqpuCircuit* circuit) {
  return circuit ? circuit_depth(Cc(circuit)->gates, Cc(circuit)->n) : 0;
}

extern "C" NqpuError nqpu_circuit_plan_stats(const NqpuCircuit* circuit, uint32_t num_qubits,
                                             NqpuDtype dtype, NqpuMode mode, uint64_t* out, uint32_t len) {
  if (!circuit || !out) return NQPU_NULL_POINTER;
  if (len < 3) return NQPU_INVALID_PARAMETER;
  const CircuitImpl* c = Cc(circuit);
  if (num_qubits < c->n || num_qubits > uint32_t(kMaxQubits)) return NQPU_INVALID_PARAMETER;
  if (!mode_ok(mode)) return NQPU_INVALID_PARAMETER;
  PlanStats st;
  if (!circuit_plan_stats(c, num_qubits, dtype == NQPU_C64 ? DType::C64 : DType::C128, int(mode), &st))
    return NQPU_INVALID_PARAMETER;
  out[0] = st.passes;
  out[1] = st.ops;
  out[2] = st.stages;
  if (len >= 4) out[3] = st.upload_bytes;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_circuit_auto_mode(const NqpuCircuit* circuit, uint32_t num_qubits, NqpuDtype dtype,
                                            NqpuMode* out) {
  if (!circuit || !out) return NQPU_NULL_POINTER;
  const CircuitImpl* c = Cc(circuit);
  if (num_qubits < c->n || num_qubits > uint32_t(kMaxQubits)) return NQPU_INVALID_PARAMETER;
  const Segment seg = circuit_segments(c->gates).front();
  const std::vector<Op> ops =
      lower_circuit(std::vector<GateRec>(c->gates.begin() + long(seg.begin), c->gates.begin() + long(seg.end)));
  *out = NqpuMode(auto_mode_for(ops, num_qubits, dtype == NQPU_C64 ? DType::C64 : DType::C128));
  return NQPU_OK;
}

extern "C" NqpuError nqpu_tile_config_set(NqpuDtype dtype, uint32_t ctas_per_sm) {
  if (ctas_per_sm != 1 && ctas_per_sm != 2 && ctas_per_sm != 4) return NQPU_INVALID_PARAMETER;
  tile_config_set(dtype == NQPU_C64 ? DType::C64 : DType::C128, int(ctas_per_sm));
  return NQPU_OK;
}

extern "C" uint32_t nqpu_tile_config_get(NqpuDtype dtype) {
  return uint32_t(tile_config_get(dtype == NQPU_C64 ? DType::C64 : DType::C128));
}

// ---------------------------------------------------------------------------
// Utility
// ---------------------------------------------------------------------------
extern "C" NqpuVersion nqpu_version(void) {
  NqpuVersion v;
  v.major = 0;  // c_ffi.rs:1404 reports 0.1.0
  v.minor = 1;
  v.patch = 0;
  return v;
}

extern "C" const char* nqpu_error_message(NqpuError error) {
  switch (error) {
    case NQPU_OK: return "Success";
    case NQPU_INVALID_QUBIT: return "Invalid qubit index";
    case NQPU_INVALID_PARAMETER: return "Invalid parameter";
    case NQPU_ALLOCATION_FAILED: return "Memory allocation failed";
    case NQPU_SIMULATION_FAILED: return "Simulation failed";
    case NQPU_NULL_POINTER: return "Null pointer";
    case NQPU_INVALID_HANDLE: return "Invalid handle";
  }
  return "Unknown error";
}
