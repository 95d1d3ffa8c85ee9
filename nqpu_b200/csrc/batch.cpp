// Host side of batched execution: per-circuit tiled plans, the dependency-
// ordered task queue, the HBM state arena, and a captured CUDA graph that
// resets the queue, runs the persistent kernel and copies the results back.
#include <chrono>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <iterator>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nqpu_b200.h"
#include "batch.h"
#include "engine.h"
#include "kernels.h"
#include "planner.h"

namespace nqpu {

struct BatchEntry {
  int n = 0;
  std::vector<GateRec> gates;
  std::vector<double> J, h;
};

struct BatchImpl {
  std::vector<BatchEntry> entries;
  int small_max = 13;    // circuits up to this size run in one CTA's shared memory
  int plan_kmax = 13;    // tile bits of the larger circuits' passes
  int order = 0;         // queue order strategy
  int ctas_per_sm = 2;
  uint32_t spin_limit = kBatchSpinLimit;  // polls of a bounded dependency wait
  bool drop_tile = false;                 // failure injection: leave one pass-0 tile out of the queue
  bool built = false;
  cudaStream_t stream = nullptr;
  float* d_arena = nullptr;
  BatchCirc* d_circs = nullptr;
  BatchTask* d_tasks = nullptr;
  unsigned char* d_tables = nullptr;  // one allocation: passes, stages, ops, Ising terms
  PassRec* d_passes = nullptr;        // (interior pointers of d_tables)
  StageRec* d_stages = nullptr;
  TileOp<float>* d_ops = nullptr;
  double* d_obs = nullptr;
  uint32_t* d_counters = nullptr;
  double* d_partials = nullptr;
  double* d_results = nullptr;
  uint32_t* d_cursor = nullptr;
  int* d_err = nullptr;
  double* h_results = nullptr;
  int* h_err = nullptr;
  uint32_t n_tasks = 0, n_counters = 0;
  size_t arena_bytes = 0, n_small = 0, n_passes_total = 0, upload_bytes = 0;
  // host time of the last prepare() by phase (microseconds): plans, packing
  // of the tables and task queue, device allocations and uploads, capture
  uint64_t prep_us[4] = {0, 0, 0, 0};
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;  // bracket each graph replay on `stream`
  bool timed = false;
};

static void batch_release(BatchImpl* b) {
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  void* ptrs[] = {b->d_arena, b->d_circs, b->d_tasks, b->d_tables,
                  b->d_counters, b->d_partials, b->d_results, b->d_cursor, b->d_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (b->h_results) cudaFreeHost(b->h_results);
  if (b->h_err) cudaFreeHost(b->h_err);
  b->graph = nullptr;
  b->d_arena = nullptr; b->d_circs = nullptr; b->d_tasks = nullptr; b->d_tables = nullptr; b->d_passes = nullptr;
  b->d_stages = nullptr; b->d_ops = nullptr; b->d_obs = nullptr; b->d_counters = nullptr;
  b->d_partials = nullptr; b->d_results = nullptr; b->d_cursor = nullptr; b->d_err = nullptr;
  b->h_results = nullptr; b->h_err = nullptr;
  b->built = false;
}

template <typename T>
static cudaError_t upload(T** d, const T* h, size_t count) {
  const size_t bytes = std::max<size_t>(1, count) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(d), bytes);
  if (e != cudaSuccess) return e;
  if (count) e = cudaMemcpy(*d, h, count * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}
template <typename T>
static cudaError_t upload(T** d, const std::vector<T>& h) {
  return upload(d, h.data(), h.size());
}

// Host staging of the batch tables: one pinned buffer per process, grown on
// demand and kept for the process's lifetime, so a prepare() after the first
// packs into memory that is already mapped and uploads it in one DMA.  The
// mutex serialises prepares of different batches from the pack through the
// end of the upload.
struct PinnedStage {
  std::mutex mu;
  unsigned char* p = nullptr;
  size_t cap = 0;
};
static PinnedStage g_stage;

// Run f(lo, hi) over [0, n) split across up to 16 host threads.
template <typename F>
static void parallel_ranges(size_t n, size_t min_per_thread, F&& f) {
  const size_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const size_t nt = std::min(hw, std::max<size_t>(1, n / std::max<size_t>(1, min_per_thread)));
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; ++t) th.emplace_back(f, n * t / nt, n * (t + 1) / nt);
  f(size_t(0), n / nt);
  for (auto& x : th) x.join();
}

static uint64_t since_us(std::chrono::steady_clock::time_point& t) {
  const auto now = std::chrono::steady_clock::now();
  const uint64_t us = uint64_t(std::chrono::duration_cast<std::chrono::microseconds>(now - t).count());
  t = now;
  return us;
}

static cudaError_t batch_build(BatchImpl* b) {
  auto clk = std::chrono::steady_clock::now();
  batch_release(b);
  if (!b->stream) {
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
  }
  std::vector<BatchCirc> circs(b->entries.size());
  uint64_t arena_amps = 0;
  uint32_t counters = 0, partials = 0;
  b->n_small = 0;
  // per-circuit tiled plans (independent: built on host threads), then
  // concatenated with rebased stage/op indices
  const size_t nc = b->entries.size();
  std::vector<TilePlan> plans(nc);
  std::vector<char> plan_ok(nc, 0);
  parallel_ranges(nc, 64, [&](size_t lo, size_t hi) {
    for (size_t ci = lo; ci < hi; ++ci) {
      const BatchEntry& E = b->entries[ci];
      const bool small = E.n <= b->small_max;
      const int kmax = small ? 13 : std::min(b->plan_kmax, 13);
      std::string err;
      plan_ok[ci] = build_tile_plan(lower_circuit(E.gates), E.n, DType::C64, kmax, &plans[ci], &err) &&
                    (!small || plans[ci].passes.size() == 1);
    }
  });
  b->prep_us[0] = since_us(clk);
  // the concatenated tables: offsets per circuit first, then every circuit's
  // records copied (with rebased stage / op indices) on host threads into
  // arrays allocated without initialisation
  std::vector<size_t> pbase(nc + 1, 0), sbase(nc + 1, 0), obase(nc + 1, 0), jbase(nc + 1, 0);
  for (size_t ci = 0; ci < nc; ++ci) {
    if (!plan_ok[ci]) return cudaErrorInvalidValue;
    pbase[ci + 1] = pbase[ci] + plans[ci].passes.size();
    sbase[ci + 1] = sbase[ci] + plans[ci].stages.size();
    obase[ci + 1] = obase[ci] + plans[ci].ops_f.size();
    jbase[ci + 1] = jbase[ci] + b->entries[ci].J.size() + b->entries[ci].h.size();
  }
  if (sbase[nc] > size_t(INT32_MAX) || obase[nc] > size_t(INT32_MAX) || jbase[nc] > size_t(INT32_MAX))
    return cudaErrorInvalidValue;  // the device records index tables with 32-bit offsets
  auto align256 = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t off_s = align256(pbase[nc] * sizeof(PassRec));
  const size_t off_o = off_s + align256(sbase[nc] * sizeof(StageRec));
  const size_t off_j = off_o + align256(obase[nc] * sizeof(TileOp<float>));
  const size_t table_bytes = off_j + align256(std::max<size_t>(1, jbase[nc]) * sizeof(double));
  std::unique_lock<std::mutex> stage_lock(g_stage.mu);
  if (g_stage.cap < table_bytes) {
    if (g_stage.p) cudaFreeHost(g_stage.p);
    g_stage.p = nullptr;
    g_stage.cap = 0;
    cudaError_t ae = cudaHostAlloc(reinterpret_cast<void**>(&g_stage.p), table_bytes, cudaHostAllocPortable);
    if (ae != cudaSuccess) return ae;
    g_stage.cap = table_bytes;
  }
  PassRec* passes = reinterpret_cast<PassRec*>(g_stage.p);
  StageRec* stages = reinterpret_cast<StageRec*>(g_stage.p + off_s);
  TileOp<float>* ops = reinterpret_cast<TileOp<float>*>(g_stage.p + off_o);
  double* obs = reinterpret_cast<double*>(g_stage.p + off_j);
  parallel_ranges(nc, 16, [&](size_t lo, size_t hi) {
    for (size_t ci = lo; ci < hi; ++ci) {
      const TilePlan& tp = plans[ci];
      PassRec* pd = passes + pbase[ci];
      for (size_t i = 0; i < tp.passes.size(); ++i) {
        pd[i] = tp.passes[i];
        pd[i].stage_begin += int32_t(sbase[ci]);
        pd[i].stage_end += int32_t(sbase[ci]);
      }
      StageRec* sd = stages + sbase[ci];
      for (size_t i = 0; i < tp.stages.size(); ++i) {
        sd[i] = tp.stages[i];
        sd[i].op_begin += int32_t(obase[ci]);
        sd[i].op_end += int32_t(obase[ci]);
      }
      if (!tp.ops_f.empty()) std::memcpy(ops + obase[ci], tp.ops_f.data(), tp.ops_f.size() * sizeof(TileOp<float>));
      const BatchEntry& E = b->entries[ci];
      std::copy(E.J.begin(), E.J.end(), obs + jbase[ci]);
      std::copy(E.h.begin(), E.h.end(), obs + jbase[ci] + E.J.size());
    }
  });
  for (size_t ci = 0; ci < nc; ++ci) {
    const BatchEntry& E = b->entries[ci];
    BatchCirc& C = circs[ci];
    std::memset(&C, 0, sizeof(C));
    C.n = E.n;
    C.small = E.n <= b->small_max ? 1 : 0;
    const TilePlan& tp = plans[ci];
    C.pass_base = int32_t(pbase[ci]);
    C.n_passes = int32_t(tp.passes.size());
    C.obs_base = int32_t(jbase[ci]);
    C.result = int32_t(ci);
    if (C.small) {
      ++b->n_small;
    } else {
      C.amp_off = arena_amps;
      arena_amps += 1ull << E.n;
      C.done_base = int32_t(counters);
      counters += uint32_t(C.n_passes) + 1;
      C.meas_k = std::min(13, E.n);
      C.meas_tiles = 1 << (E.n - C.meas_k);
      C.part_base = int32_t(partials);
      partials += uint32_t(C.meas_tiles);
    }
  }
  b->n_passes_total = pbase[nc];
  // task queue: every task depends only on tasks queued before it.
  // Rounds r = 0, 1, ...: phase r of every large circuit (largest first; phase
  // n_passes = measurement), all its tiles.  Small circuits are spread between
  // rounds (order 0), placed first (order 1) or last (order 2).
  std::vector<int> large, small;
  for (size_t ci = 0; ci < circs.size(); ++ci) (circs[ci].small ? small : large).push_back(int(ci));
  std::stable_sort(large.begin(), large.end(), [&](int a, int c) { return circs[a].n > circs[c].n; });
  std::stable_sort(small.begin(), small.end(), [&](int a, int c) { return circs[a].n > circs[c].n; });
  int max_rounds = 0;
  for (int ci : large) max_rounds = std::max(max_rounds, circs[ci].n_passes + 1);
  std::vector<BatchTask> tasks;
  size_t si = 0;
  auto push_small = [&](size_t upto) {
    for (; si < std::min(upto, small.size()); ++si) tasks.push_back(BatchTask{small[si], -1, 0, 0});
  };
  if (b->order == 1) push_small(small.size());
  bool dropped = false;
  for (int r = 0; r < max_rounds; ++r) {
    for (int ci : large) {
      const BatchCirc& C = circs[ci];
      if (r > C.n_passes) continue;
      const uint32_t tiles = r < C.n_passes ? (1u << passes[C.pass_base + r].n_out) : uint32_t(C.meas_tiles);
      for (uint32_t t = 0; t < tiles; ++t) {
        // failure injection (tests): the first tile of the first large
        // circuit's first pass is never queued, so that circuit's pass-1
        // tiles wait on a counter that cannot complete and their bounded
        // waits expire
        if (b->drop_tile && !dropped && r == 0) {
          dropped = true;
          continue;
        }
        tasks.push_back(BatchTask{ci, r, t, 0});
      }
    }
    if (b->order == 0) push_small(small.size() * size_t(r + 1) / size_t(max_rounds));
  }
  push_small(small.size());
  b->n_tasks = uint32_t(tasks.size());
  b->n_counters = std::max<uint32_t>(1, counters);
  b->arena_bytes = size_t(arena_amps) * 8;

  b->prep_us[1] = since_us(clk);
  cudaError_t e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_arena), std::max<size_t>(16, b->arena_bytes))) != cudaSuccess) return e;
  if ((e = upload(&b->d_circs, circs)) != cudaSuccess) return e;
  if ((e = upload(&b->d_tasks, tasks)) != cudaSuccess) return e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_tables), table_bytes)) != cudaSuccess) return e;
  b->d_passes = reinterpret_cast<PassRec*>(b->d_tables);
  b->d_stages = reinterpret_cast<StageRec*>(b->d_tables + off_s);
  b->d_ops = reinterpret_cast<TileOp<float>*>(b->d_tables + off_o);
  b->d_obs = reinterpret_cast<double*>(b->d_tables + off_j);
  if ((e = cudaMemcpyAsync(b->d_tables, g_stage.p, table_bytes, cudaMemcpyHostToDevice, b->stream)) != cudaSuccess)
    return e;
  // the staging buffer is free for the next prepare once its copy is done
  if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return e;
  stage_lock.unlock();
  b->upload_bytes = circs.size() * sizeof(BatchCirc) + tasks.size() * sizeof(BatchTask) +
                    pbase[nc] * sizeof(PassRec) + sbase[nc] * sizeof(StageRec) +
                    obase[nc] * sizeof(TileOp<float>) + jbase[nc] * sizeof(double);
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_counters), sizeof(uint32_t) * b->n_counters)) != cudaSuccess) return e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_partials), sizeof(double) * std::max<uint32_t>(1, partials))) != cudaSuccess) return e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_results), sizeof(double) * std::max<size_t>(1, circs.size()))) != cudaSuccess) return e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_cursor), sizeof(uint32_t))) != cudaSuccess) return e;
  if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_err), sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(reinterpret_cast<void**>(&b->h_results), sizeof(double) * std::max<size_t>(1, circs.size()))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(reinterpret_cast<void**>(&b->h_err), sizeof(int))) != cudaSuccess) return e;

  b->prep_us[2] = since_us(clk);
  // capture: reset counters/cursor/error, the persistent launch, result copies
  BatchLaunch L;
  L.arena = b->d_arena; L.circs = b->d_circs; L.tasks = b->d_tasks; L.n_tasks = b->n_tasks;
  L.passes = b->d_passes; L.stages = b->d_stages; L.ops = b->d_ops; L.obs = b->d_obs;
  L.counters = b->d_counters; L.partials = b->d_partials; L.results = b->d_results;
  L.cursor = b->d_cursor; L.err = b->d_err;
  L.grid = unsigned(std::max(1, device_sms() * b->ctas_per_sm));
  L.spin_limit = b->spin_limit;
  // warm the module and the smem attribute outside the capture
  if ((e = cudaMemsetAsync(b->d_cursor, 0xFF, sizeof(uint32_t), b->stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream)) != cudaSuccess) return e;
  BatchLaunch warm = L;
  warm.n_tasks = 0;
  warm.grid = 1;
  if ((e = launch_batch(warm, b->stream)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return e;
  cudaGraph_t g;
  if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
  cudaMemsetAsync(b->d_counters, 0, sizeof(uint32_t) * b->n_counters, b->stream);
  cudaMemsetAsync(b->d_cursor, 0, sizeof(uint32_t), b->stream);
  cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream);
  launch_batch(L, b->stream);
  cudaMemcpyAsync(b->h_results, b->d_results, sizeof(double) * circs.size(), cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(b->h_err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
  if ((e = cudaStreamEndCapture(b->stream, &g)) != cudaSuccess) return e;
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return e;
  b->prep_us[3] = since_us(clk);
  b->built = true;
  return cudaSuccess;
}

}  // namespace nqpu

using namespace nqpu;

static BatchImpl* B(NqpuBatch* h) { return reinterpret_cast<BatchImpl*>(h); }

extern "C" NqpuBatch* nqpu_batch_create(void) {
  if (!device_ready()) return nullptr;
  auto* b = new (std::nothrow) BatchImpl();
  return reinterpret_cast<NqpuBatch*>(b);
}

extern "C" void nqpu_batch_destroy(NqpuBatch* batch) {
  if (!batch) return;
  BatchImpl* b = B(batch);
  batch_release(b);
  if (b->ev_begin) cudaEventDestroy(b->ev_begin);
  if (b->ev_end) cudaEventDestroy(b->ev_end);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

extern "C" NqpuError nqpu_batch_add_ising(NqpuBatch* batch, const NqpuCircuit* circuit, const double* J,
                                          const double* h, uint32_t* index) {
  if (!batch || !circuit || !h) return NQPU_NULL_POINTER;
  const CircuitImpl* c = reinterpret_cast<const CircuitImpl*>(circuit);
  if (c->n < 5 || c->n > 24) return NQPU_INVALID_PARAMETER;  // batched circuits: 5..24 qubits (3 bond tables)
  if (circuit_has_mid(c->gates)) return NQPU_INVALID_PARAMETER;  // measurement-free circuits only
  if (c->n > 1 && !J) return NQPU_NULL_POINTER;
  BatchImpl* b = B(batch);
  BatchEntry e;
  e.n = int(c->n);
  e.gates = c->gates;
  e.J.assign(J, J + (c->n - 1));
  e.h.assign(h, h + c->n);
  if (index) *index = uint32_t(b->entries.size());
  b->entries.push_back(std::move(e));
  b->built = false;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_batch_add_ising_arrays(NqpuBatch* batch, uint32_t count, const uint32_t* num_qubits,
                                                 const uint64_t* gate_offsets, const uint32_t* codes,
                                                 const int32_t* qubits, const double* params,
                                                 const NqpuComplex* matrices, const double* J, const double* h,
                                                 uint32_t* first_index) {
  if (!batch) return NQPU_NULL_POINTER;
  if (count == 0) return NQPU_OK;
  if (!num_qubits || !gate_offsets || !h || !J) return NQPU_NULL_POINTER;
  BatchImpl* b = B(batch);
  // each circuit's first J and h entry (J: n - 1 bonds, h: n sites)
  std::vector<size_t> jo(size_t(count) + 1, 0), ho(size_t(count) + 1, 0);
  for (uint32_t i = 0; i < count; ++i) {
    if (num_qubits[i] < 5 || num_qubits[i] > 24) return NQPU_INVALID_PARAMETER;
    if (gate_offsets[i + 1] < gate_offsets[i]) return NQPU_INVALID_PARAMETER;
    jo[i + 1] = jo[i] + (num_qubits[i] - 1);
    ho[i + 1] = ho[i] + num_qubits[i];
  }
  std::vector<BatchEntry> add(count);
  std::vector<NqpuError> errs(count, NQPU_OK);
  parallel_ranges(count, 64, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) {
      CircuitImpl tmp;
      tmp.n = num_qubits[i];
      const uint64_t g0 = gate_offsets[i], g1 = gate_offsets[i + 1];
      NqpuError e = circuit_append_gates(&tmp, codes ? codes + g0 : nullptr, qubits ? qubits + 3 * g0 : nullptr,
                                         params ? params + 4 * g0 : nullptr, matrices ? matrices + 16 * g0 : nullptr,
                                         size_t(g1 - g0));
      if (e == NQPU_OK && circuit_has_mid(tmp.gates)) e = NQPU_INVALID_PARAMETER;  // measurement-free only
      errs[i] = e;
      if (e != NQPU_OK) continue;
      BatchEntry& E = add[i];
      E.n = int(num_qubits[i]);
      E.gates = std::move(tmp.gates);
      E.J.assign(J + jo[i], J + jo[i + 1]);
      E.h.assign(h + ho[i], h + ho[i + 1]);
    }
  });
  for (NqpuError e : errs)
    if (e != NQPU_OK) return e;  // the batch is unchanged
  if (first_index) *first_index = uint32_t(b->entries.size());
  b->entries.insert(b->entries.end(), std::make_move_iterator(add.begin()), std::make_move_iterator(add.end()));
  b->built = false;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_batch_config(NqpuBatch* batch, NqpuBatchParam param, int32_t value) {
  if (!batch) return NQPU_NULL_POINTER;
  BatchImpl* b = B(batch);
  switch (param) {
    case NQPU_BATCH_SMALL_MAX_QUBITS:
      if (value < 5 || value > 13) return NQPU_INVALID_PARAMETER;
      b->small_max = value;
      break;
    case NQPU_BATCH_TILE_QUBITS:
      if (value < 10 || value > 13) return NQPU_INVALID_PARAMETER;
      b->plan_kmax = value;
      break;
    case NQPU_BATCH_QUEUE_ORDER:
      if (value < 0 || value > 2) return NQPU_INVALID_PARAMETER;
      b->order = value;
      break;
    case NQPU_BATCH_CTAS_PER_SM:
      if (value < 1 || value > 2) return NQPU_INVALID_PARAMETER;
      b->ctas_per_sm = value;
      break;
    case NQPU_BATCH_SPIN_LIMIT:
      if (value < 1) return NQPU_INVALID_PARAMETER;
      b->spin_limit = uint32_t(value);
      break;
    case NQPU_BATCH_DROP_TILE:
      if (value < 0 || value > 1) return NQPU_INVALID_PARAMETER;
      b->drop_tile = value == 1;
      break;
    default:
      return NQPU_INVALID_PARAMETER;
  }
  b->built = false;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_batch_prepare(NqpuBatch* batch) {
  if (!batch) return NQPU_NULL_POINTER;
  BatchImpl* b = B(batch);
  if (b->entries.empty()) return NQPU_INVALID_PARAMETER;
  const cudaError_t e = batch_build(b);
  if (e == cudaErrorMemoryAllocation) return NQPU_ALLOCATION_FAILED;
  if (e == cudaErrorInvalidValue) return NQPU_INVALID_PARAMETER;
  return e == cudaSuccess ? NQPU_OK : NQPU_SIMULATION_FAILED;
}

extern "C" NqpuError nqpu_batch_run(NqpuBatch* batch, double* results, uint32_t len) {
  if (!batch || !results) return NQPU_NULL_POINTER;
  BatchImpl* b = B(batch);
  if (len < b->entries.size()) return NQPU_INVALID_PARAMETER;
  if (!b->built) {
    NqpuError pe = nqpu_batch_prepare(batch);
    if (pe != NQPU_OK) return pe;
  }
  if (!b->ev_begin && (cudaEventCreate(&b->ev_begin) != cudaSuccess || cudaEventCreate(&b->ev_end) != cudaSuccess))
    return NQPU_SIMULATION_FAILED;
  if (cudaEventRecord(b->ev_begin, b->stream) != cudaSuccess) return NQPU_SIMULATION_FAILED;
  if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return NQPU_SIMULATION_FAILED;
  if (cudaEventRecord(b->ev_end, b->stream) != cudaSuccess) return NQPU_SIMULATION_FAILED;
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return NQPU_SIMULATION_FAILED;
  b->timed = true;
  if (*b->h_err != 0) return NQPU_SIMULATION_FAILED;  // a bounded wait expired
  std::memcpy(results, b->h_results, sizeof(double) * b->entries.size());
  return NQPU_OK;
}

extern "C" NqpuError nqpu_batch_stats(const NqpuBatch* batch, uint64_t* out, uint32_t len) {
  if (!batch || !out) return NQPU_NULL_POINTER;
  if (len < 5) return NQPU_INVALID_PARAMETER;
  const BatchImpl* b = reinterpret_cast<const BatchImpl*>(batch);
  out[0] = b->entries.size();
  out[1] = b->n_small;
  out[2] = b->n_tasks;
  out[3] = b->arena_bytes;
  out[4] = b->n_passes_total;
  if (len >= 6) out[5] = b->upload_bytes;
  for (uint32_t i = 0; i < 4 && 6 + i < len; ++i) out[6 + i] = b->prep_us[i];
  return NQPU_OK;
}

extern "C" NqpuError nqpu_batch_last_run_ms(const NqpuBatch* batch, float* ms) {
  if (!batch || !ms) return NQPU_NULL_POINTER;
  const BatchImpl* b = reinterpret_cast<const BatchImpl*>(batch);
  if (!b->timed) return NQPU_INVALID_PARAMETER;
  return cudaEventElapsedTime(ms, b->ev_begin, b->ev_end) == cudaSuccess ? NQPU_OK : NQPU_SIMULATION_FAILED;
}
