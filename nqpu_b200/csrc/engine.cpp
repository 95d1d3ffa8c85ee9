// Engine objects: device context, state allocation, reductions glue and the
// circuit runner (tiled passes / per-gate / fused).
#include "engine.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include "device_once.h"
#include "fused.h"
#include "kernels.h"
#include "tcpass.h"
#include "tcrun.h"

namespace nqpu {

namespace {
std::once_flag g_dev_once;
bool g_dev_ok = false;

void dev_init() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    g_dev_ok = false;
    return;
  }
  g_dev_ok = true;
}
}  // namespace

bool device_ready() {
  std::call_once(g_dev_once, dev_init);
  return g_dev_ok;
}

// SM count of the current device (grids are sized in multiples of it), read
// once per device.
int device_sms() {
  static PerDeviceOnce<int> sms;
  int dev = 0;
  if (!device_ready() || cudaGetDevice(&dev) != cudaSuccess) return 148;
  return sms.get(dev, [dev] {
    int v = 0;
    return (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0) ? v : 148;
  }, 148);
}

StateImpl* state_new(uint32_t n, DType dt) {
  if (!device_ready()) return nullptr;
  auto* s = new (std::nothrow) StateImpl();
  if (!s) return nullptr;
  s->n = n;
  s->dt = dt;
  s->bytes = size_t(amp_bytes(dt)) << n;
  bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc(&s->amp, s->bytes) == cudaSuccess;
  ok = ok && cudaMalloc(reinterpret_cast<void**>(&s->scratch), reduce_scratch_bytes(int(n))) == cudaSuccess;
  ok = ok && cudaMalloc(reinterpret_cast<void**>(&s->d_small), 512 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMallocHost(reinterpret_cast<void**>(&s->h_small), 512 * sizeof(double)) == cudaSuccess;
  ok = ok && launch_set_basis(dt, s->amp, int(n), 0, s->stream, device_sms()) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(s->stream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    state_free(s);
    return nullptr;
  }
  return s;
}

void state_free(StateImpl* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->amp) cudaFree(s->amp);
  if (s->scratch) cudaFree(s->scratch);
  if (s->d_small) cudaFree(s->d_small);
  if (s->h_small) cudaFreeHost(s->h_small);
  if (s->d_uni) cudaFree(s->d_uni);
  if (s->d_shots) cudaFree(s->d_shots);
  if (s->run_norm) cudaFree(s->run_norm);
  if (s->run_err) cudaFree(s->run_err);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

cudaError_t state_run_scratch(StateImpl* s, size_t doubles, double** norm, int** err) {
  cudaError_t e;
  if (s->run_norm_cap < doubles) {
    // the old buffer may back a run still queued on the state's stream
    if (s->run_norm && (e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return e;
    if (s->run_norm) cudaFree(s->run_norm);
    s->run_norm = nullptr;
    s->run_norm_cap = 0;
    if ((e = cudaMalloc(reinterpret_cast<void**>(&s->run_norm), doubles * sizeof(double))) != cudaSuccess) return e;
    s->run_norm_cap = doubles;
  }
  if (!s->run_err && (e = cudaMalloc(reinterpret_cast<void**>(&s->run_err), sizeof(int))) != cudaSuccess) return e;
  // the expiry flag of an earlier run is cleared, so this run reports its own
  if ((e = cudaMemsetAsync(s->run_err, 0, sizeof(int), s->stream)) != cudaSuccess) return e;
  *norm = s->run_norm;
  *err = s->run_err;
  return cudaSuccess;
}

cudaError_t state_run_error(StateImpl* s) {
  if (!s->run_err) return cudaSuccess;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, s->run_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return e;
  return h ? cudaErrorLaunchTimeout : cudaSuccess;
}

cudaError_t state_zsums(const StateImpl* s, double* zs, double* total) {
  const int n = int(s->n);
  cudaError_t e = launch_zsums(s->dt, s->amp, n, s->scratch, s->d_small, s->stream, device_sms());
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(s->h_small, s->d_small, sizeof(double) * (n + 1), cudaMemcpyDeviceToHost, s->stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return e;
  if (zs) std::memcpy(zs, s->h_small, sizeof(double) * (n + 1));
  if (total) *total = s->h_small[0];
  return cudaSuccess;
}

cudaError_t state_measure(StateImpl* s, uint32_t qubit, uint32_t* outcome, double* probability) {
  std::vector<double> z(s->n + 1);
  cudaError_t e = state_zsums(s, z.data(), nullptr);
  if (e != cudaSuccess) return e;
  const double prob0 = z[0] - z[1 + qubit];  // sum over bit q == 0
  const double prob1 = 1.0 - prob0;          // c_ffi.rs:546
  const double r = next_random_f64();
  const uint32_t out = r < prob0 ? 0u : 1u;
  const double po = out == 0 ? prob0 : prob1;
  const double renorm = 1.0 / std::sqrt(po);
  e = launch_collapse(s->dt, s->amp, int(s->n), int(qubit), int(out), renorm, s->stream, device_sms());
  if (e != cudaSuccess) return e;
  *outcome = out;
  if (probability) *probability = po;
  return cudaSuccess;
}

cudaError_t state_reset_qubit(StateImpl* s, uint32_t qubit) {
  std::vector<double> z(s->n + 1);
  cudaError_t e = state_zsums(s, z.data(), nullptr);
  if (e != cudaSuccess) return e;
  const double keep = z[0] - z[1 + qubit];  // norm of the |0> half
  const double f = keep > 0.0 ? 1.0 / std::sqrt(keep) : 1.0;
  return launch_collapse(s->dt, s->amp, int(s->n), int(qubit), 0, f, s->stream, device_sms());
}

cudaError_t state_pauli(const StateImpl* s, uint64_t xm, uint64_t zm, uint64_t ym, double* out2) {
  cudaError_t e = launch_pauli(s->dt, s->amp, int(s->n), xm, zm, ym, s->scratch, s->d_small, s->stream, device_sms());
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(s->h_small, s->d_small, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return e;
  out2[0] = s->h_small[0];
  out2[1] = s->h_small[1];
  return cudaSuccess;
}

cudaError_t state_inner(const StateImpl* a, const StateImpl* b, double* out2) {
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return e;
  e = launch_inner(a->dt, a->amp, b->dt, b->amp, int(a->n), a->scratch, a->d_small, a->stream, device_sms());
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(a->h_small, a->d_small, 2 * sizeof(double), cudaMemcpyDeviceToHost, a->stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return e;
  out2[0] = a->h_small[0];
  out2[1] = a->h_small[1];
  return cudaSuccess;
}

cudaError_t state_sample(const StateImpl* sc, const double* uniforms, uint32_t shots, uint64_t* out) {
  StateImpl* s = const_cast<StateImpl*>(sc);
  cudaError_t e;
  if (s->shot_cap < shots) {
    e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return e;
    if (s->d_uni) cudaFree(s->d_uni);
    if (s->d_shots) cudaFree(s->d_shots);
    s->d_uni = nullptr;
    s->d_shots = nullptr;
    s->shot_cap = 0;
    if ((e = cudaMalloc(reinterpret_cast<void**>(&s->d_uni), sizeof(double) * shots)) != cudaSuccess) return e;
    if ((e = cudaMalloc(reinterpret_cast<void**>(&s->d_shots), sizeof(uint64_t) * shots)) != cudaSuccess) return e;
    s->shot_cap = shots;
  }
  if ((e = cudaMemcpyAsync(s->d_uni, uniforms, sizeof(double) * shots, cudaMemcpyHostToDevice, s->stream)) != cudaSuccess) return e;
  if ((e = launch_sample(s->dt, s->amp, int(s->n), s->d_uni, shots, s->scratch, s->d_shots, s->stream, device_sms())) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(out, s->d_shots, sizeof(uint64_t) * shots, cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s->stream);
}

// Probabilities in chunks through a device buffer (the full 2^n FP64 vector may
// not fit next to the state).
cudaError_t state_probabilities(const StateImpl* s, double* out) {
  const uint64_t dim = 1ull << s->n;
  const uint64_t chunk = std::min<uint64_t>(dim, 1ull << 24);
  double* d = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&d), chunk * sizeof(double));
  if (e != cudaSuccess) return e;
  const size_t ab = amp_bytes(s->dt);
  for (uint64_t off = 0; off < dim && e == cudaSuccess; off += chunk) {
    const uint64_t cnt = std::min(chunk, dim - off);
    e = launch_probabilities(s->dt, static_cast<const char*>(s->amp) + off * ab, cnt, d, s->stream, device_sms());
    if (e == cudaSuccess) e = cudaMemcpyAsync(out + off, d, cnt * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  }
  cudaFree(d);
  return e;
}

cudaError_t state_download_c128(const StateImpl* s, NqpuComplex* out) {
  const uint64_t dim = 1ull << s->n;
  if (s->dt == DType::C128) {
    cudaError_t e = cudaMemcpyAsync(out, s->amp, dim * 16, cudaMemcpyDeviceToHost, s->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s->stream);
  }
  const uint64_t chunk = std::min<uint64_t>(dim, 1ull << 22);
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, chunk * 16);
  if (e != cudaSuccess) return e;
  for (uint64_t off = 0; off < dim && e == cudaSuccess; off += chunk) {
    const uint64_t cnt = std::min(chunk, dim - off);
    e = launch_convert(DType::C64, static_cast<const char*>(s->amp) + off * 8, DType::C128, d, cnt, s->stream, device_sms());
    if (e == cudaSuccess) e = cudaMemcpyAsync(out + off, d, cnt * 16, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  }
  cudaFree(d);
  return e;
}

cudaError_t state_upload_c128(StateImpl* s, const NqpuComplex* in) {
  const uint64_t dim = 1ull << s->n;
  if (s->dt == DType::C128) {
    cudaError_t e = cudaMemcpyAsync(s->amp, in, dim * 16, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s->stream);
  }
  const uint64_t chunk = std::min<uint64_t>(dim, 1ull << 22);
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, chunk * 16);
  if (e != cudaSuccess) return e;
  for (uint64_t off = 0; off < dim && e == cudaSuccess; off += chunk) {
    const uint64_t cnt = std::min(chunk, dim - off);
    e = cudaMemcpyAsync(d, in + off, cnt * 16, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = launch_convert(DType::C128, d, DType::C64, static_cast<char*>(s->amp) + off * 8, cnt, s->stream, device_sms());
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  }
  cudaFree(d);
  return e;
}

// ---------------------------------------------------------------------------
// Circuits
// ---------------------------------------------------------------------------
static void plan_free(DevicePlan* p) {
  if (!p) return;
  if (p->d_passes) cudaFree(p->d_passes);
  if (p->d_stages) cudaFree(p->d_stages);
  if (p->d_ops) cudaFree(p->d_ops);
  if (p->fused) fused_plan_free(p->fused);
  if (p->tc) tc_plan_free(p->tc);
  delete p;
}

void circuit_free(CircuitImpl* c) {
  if (!c) return;
  cudaDeviceSynchronize();
  for (auto& kv : c->plans) plan_free(kv.second);
  delete c;
}

bool circuit_has_mid(const std::vector<GateRec>& gates) {
  for (const GateRec& g : gates)
    if (gate_is_mid(g.code)) return true;
  return false;
}

std::vector<Segment> circuit_segments(const std::vector<GateRec>& gates) {
  std::vector<Segment> segs;
  size_t b = 0;
  for (size_t i = 0; i < gates.size(); ++i)
    if (gate_is_mid(gates[i].code)) {
      segs.push_back(Segment{b, i, long(i)});
      b = i + 1;
    }
  segs.push_back(Segment{b, gates.size(), -1});
  return segs;
}

static bool plan_host(const CircuitImpl* c, const Segment& seg, uint32_t n, DType dt, int mode, DevicePlan* p) {
  p->ops = lower_circuit(std::vector<GateRec>(c->gates.begin() + long(seg.begin), c->gates.begin() + long(seg.end)));
  p->stats = PlanStats{};
  if (mode == NQPU_MODE_TILED && int(n) >= tile_min_qubits(dt)) {
    std::string err;
    p->kmax = tile_kmax_for(dt);
    if (!build_tile_plan(p->ops, int(n), dt, p->kmax, &p->tile, &err)) return false;
    p->stats = p->tile.stats;
  } else if (mode == NQPU_MODE_FUSED) {
    p->stats.ops = p->ops.size();
    return fused_plan_build(p->ops, int(n), dt, &p->fused, &p->stats);
  } else if (mode == NQPU_MODE_TENSOR) {
    return tc_plan_build(p->ops, int(n), dt, &p->tc, &p->stats);
  } else {
    p->stats.passes = p->ops.size();
    p->stats.ops = p->ops.size();
  }
  return true;
}

// NQPU_MODE_AUTO: the engine mode with the lower modelled device time (the
// counterpart of the reference's runtime-estimate backend choice,
// select_backend_estimated, backends/runtime/auto_simulator.rs:1452, among
// its statevector variants).  The model is in units of one HBM pass over the
// state (2 S bytes).  Tiled passes: per pass one unit plus its launch cost,
// plus the shared-memory tile work of each op (dense 1-qubit 0.15, dense
// 2-qubit 0.30, diagonal 0.058, permutations free: they are deferred into the
// write-back addresses).  Tensor passes: per pass one unit plus its launch
// cost, plus 0.35 per fused unitary (its MMAs and epilogue on every tile).
// The launch cost is about 15 us per pass in either mode (launch, pass-table
// prologue, grid tail), i.e. 15 us / (2 S / 6.5 TB/s) units: negligible at 30
// qubits, dominant below 20, where the mode with fewer passes wins.  The
// per-op coefficients are fits to 30-qubit complex64 runs of the brickwork
// (tiled 69 passes / 1200 U3, tensor 81 passes / 178 unitaries) and of the
// QFT (tiled 8 passes / 30 H + 435 controlled phases) against the copy time
// of the state.  The tensor mode is taken when its model is at least 10 %
// below the tiled one.
int auto_mode_for(const std::vector<Op>& ops, uint32_t n, DType dt) {
  if (dt != DType::C64 || int(n) < kTcMinQubits) return NQPU_MODE_TILED;
  PlanStats ts;
  if (!tc_plan_stats(ops, int(n), dt, &ts)) return NQPU_MODE_TILED;
  TilePlan tp;
  std::string err;
  if (!build_tile_plan(ops, int(n), dt, tile_kmax_for(dt), &tp, &err)) return NQPU_MODE_TENSOR;
  double work = 0.0;
  for (const Op& op : ops) {
    switch (op.kind) {
      case OP_U1: work += 0.15; break;
      case OP_U2: work += 0.30; break;
      case OP_D1:
      case OP_D2:
      case OP_PH: work += 0.058; break;
      default: break;  // OP_X1, OP_SW
    }
  }
  const double pass_us = 2.0 * std::ldexp(8.0, int(n)) / 6.5e6;  // 2 S bytes at 6.5 TB/s, in microseconds
  const double per_pass = 1.0 + 15.0 / pass_us;
  const double tiled = double(tp.stats.passes) * per_pass + work;
  const double tensor = double(ts.passes) * per_pass + 0.35 * double(ts.stages);
  return tensor < 0.9 * tiled ? NQPU_MODE_TENSOR : NQPU_MODE_TILED;
}

static std::vector<Op> segment_ops(const CircuitImpl* c, const Segment& seg) {
  return lower_circuit(std::vector<GateRec>(c->gates.begin() + long(seg.begin), c->gates.begin() + long(seg.end)));
}

bool circuit_plan_stats(const CircuitImpl* c, uint32_t n, DType dt, int mode, PlanStats* out) {
  *out = PlanStats{};
  for (const Segment& seg : circuit_segments(c->gates)) {
    DevicePlan p;
    PlanStats st;
    if (mode == NQPU_MODE_AUTO) {
      if (seg.begin == seg.end) continue;
      const int m = auto_mode_for(segment_ops(c, seg), n, dt);
      CircuitImpl one;
      one.n = c->n;
      one.gates.assign(c->gates.begin() + long(seg.begin), c->gates.begin() + long(seg.end));
      if (!circuit_plan_stats(&one, n, dt, m, &st)) return false;
      out->passes += st.passes;
      out->ops += st.ops;
      out->stages += st.stages;
      out->upload_bytes += st.upload_bytes;
      continue;
    }
    if (mode == NQPU_MODE_FUSED || mode == NQPU_MODE_TENSOR) {
      p.ops = lower_circuit(std::vector<GateRec>(c->gates.begin() + long(seg.begin), c->gates.begin() + long(seg.end)));
      const bool ok = mode == NQPU_MODE_FUSED ? fused_plan_stats(p.ops, int(n), dt, &st)
                                              : tc_plan_stats(p.ops, int(n), dt, &st);
      if (!ok) return false;
    } else {
      if (!plan_host(c, seg, n, dt, mode, &p)) return false;
      st = p.stats;
    }
    out->passes += st.passes;
    out->ops += st.ops;
    out->stages += st.stages;
    out->upload_bytes += st.upload_bytes;
  }
  return true;
}

cudaError_t run_ops_pergate(StateImpl* s, const std::vector<Op>& ops) {
  for (const Op& op : ops) {
    cudaError_t e = launch_pergate(s->dt, s->amp, int(s->n), op, s->stream, device_sms());
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static cudaError_t upload_tile(DevicePlan* p) {
  const TilePlan& t = p->tile;
  cudaError_t e;
  const size_t np = std::max<size_t>(1, t.passes.size());
  const size_t ns = std::max<size_t>(1, t.stages.size());
  const size_t opsz = t.dt == DType::C64 ? sizeof(TileOp<float>) : sizeof(TileOp<double>);
  const size_t nops = t.dt == DType::C64 ? t.ops_f.size() : t.ops_d.size();
  if ((e = cudaMalloc(reinterpret_cast<void**>(&p->d_passes), np * sizeof(PassRec))) != cudaSuccess) return e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&p->d_stages), ns * sizeof(StageRec))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&p->d_ops, std::max<size_t>(1, nops) * opsz)) != cudaSuccess) return e;
  if (!t.passes.empty() && (e = cudaMemcpy(p->d_passes, t.passes.data(), t.passes.size() * sizeof(PassRec), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  if (!t.stages.empty() && (e = cudaMemcpy(p->d_stages, t.stages.data(), t.stages.size() * sizeof(StageRec), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  if (nops) {
    const void* src = t.dt == DType::C64 ? static_cast<const void*>(t.ops_f.data()) : static_cast<const void*>(t.ops_d.data());
    if ((e = cudaMemcpy(p->d_ops, src, nops * opsz, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static cudaError_t mark(std::vector<cudaEvent_t>* ev, cudaStream_t st) {
  if (!ev) return cudaSuccess;
  cudaEvent_t e;
  cudaError_t r = cudaEventCreate(&e);
  if (r != cudaSuccess) return r;
  ev->push_back(e);
  return cudaEventRecord(e, st);
}

static cudaError_t segment_run(CircuitImpl* c, const Segment& seg, int si, StateImpl* s, int mode,
                               std::vector<cudaEvent_t>* events);

cudaError_t circuit_run(CircuitImpl* c, StateImpl* s, int mode, std::vector<cudaEvent_t>* events,
                        std::vector<uint32_t>* outcomes) {
  std::lock_guard<std::mutex> lk(c->mu);
  const std::vector<Segment> segs = circuit_segments(c->gates);
  for (size_t si = 0; si < segs.size(); ++si) {
    const Segment& seg = segs[si];
    cudaError_t e = segment_run(c, seg, int(si), s, mode, events);
    if (e != cudaSuccess) return e;
    if (seg.mid < 0) break;
    const GateRec& g = c->gates[size_t(seg.mid)];
    if (g.code == G_MEASURE) {
      uint32_t out = 0;
      if ((e = state_measure(s, uint32_t(g.q[0]), &out, nullptr)) != cudaSuccess) return e;
      if (outcomes) outcomes->push_back(out);
    } else {
      // OpenQASM reset: measure (one RNG draw) and flip the qubit back to |0>
      // when it came out 1 (the state API's nqpu_gate_reset_qubit keeps the
      // reference's projection, GateOperations::reset_qubit)
      uint32_t out = 0;
      if ((e = state_measure(s, uint32_t(g.q[0]), &out, nullptr)) != cudaSuccess) return e;
      if (out == 1) {
        Op x;
        x.kind = OP_X1;
        x.t0 = int8_t(g.q[0]);
        if ((e = launch_pergate(s->dt, s->amp, int(s->n), x, s->stream, device_sms())) != cudaSuccess) return e;
      }
    }
  }
  return cudaSuccess;
}

static cudaError_t segment_run(CircuitImpl* c, const Segment& seg, int si, StateImpl* s, int mode,
                               std::vector<cudaEvent_t>* events) {
  if (seg.begin == seg.end) return cudaSuccess;
  if (mode == NQPU_MODE_AUTO) {
    std::pair<uint64_t, int>& am = c->auto_modes[std::make_tuple(s->n, int(s->dt), si)];
    if (am.first != c->version + 1) am = {c->version + 1, auto_mode_for(segment_ops(c, seg), s->n, s->dt)};
    mode = am.second;
  }
  const int effective = (mode == NQPU_MODE_TILED && int(s->n) < tile_min_qubits(s->dt)) ? int(NQPU_MODE_PERGATE) : mode;
  const auto key = std::make_tuple(s->n, int(s->dt), effective, si);
  DevicePlan*& p = c->plans[key];
  // rebuild when the circuit changed or the tiled kernel's tile size did
  if (p && (p->version != c->version || (effective == NQPU_MODE_TILED && p->kmax != tile_kmax_for(s->dt)))) {
    cudaStreamSynchronize(s->stream);
    plan_free(p);
    p = nullptr;
  }
  if (!p) {
    p = new DevicePlan();
    if (!plan_host(c, seg, s->n, s->dt, effective, p)) {
      plan_free(p);
      p = nullptr;
      return cudaErrorInvalidValue;
    }
    if (effective == NQPU_MODE_TILED) {
      cudaError_t e = upload_tile(p);
      if (e != cudaSuccess) {
        plan_free(p);
        p = nullptr;
        return e;
      }
    }
    p->version = c->version;
  }
  cudaError_t e = mark(events, s->stream);
  if (e != cudaSuccess) return e;
  if (effective == NQPU_MODE_PERGATE) {
    for (const Op& op : p->ops) {
      if ((e = launch_pergate(s->dt, s->amp, int(s->n), op, s->stream, device_sms())) != cudaSuccess) return e;
      if ((e = mark(events, s->stream)) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  if (effective == NQPU_MODE_FUSED) {
    e = fused_run(p->fused, s, events);
    if (e != cudaSuccess) return e;
    return state_run_error(s);  // bounded-wait expiry flag
  }
  if (effective == NQPU_MODE_TENSOR) {
    e = tc_run(p->tc, s, events);
    if (e != cudaSuccess) return e;
    return state_run_error(s);  // bounded-wait expiry flag
  }
  for (size_t i = 0; i < p->tile.passes.size(); ++i) {
    e = launch_tile_pass(s->dt, s->amp, int(s->n), p->tile.passes[i], p->d_passes, p->d_stages,
                         p->d_ops, int(i), s->stream, device_sms());
    if (e != cudaSuccess) return e;
    if ((e = mark(events, s->stream)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace nqpu
