// Request loop for serving circuits of mixed sizes on one GPU.
//
// Requests (a circuit plus "all <Z_i>" or "k shots") are submitted from any
// host thread and run on complex64 states that stay resident in HBM for the
// life of the request.  A worker thread owns the device side:
//   * HBM budget: one arena of the configured size is allocated up front and
//     carved by a buddy allocator into power-of-two blocks, so a request's
//     state (2^n x 8 B, itself a power of two) costs exactly its footprint and
//     freed blocks coalesce again.
//   * Lanes: a fixed set of CUDA streams.  A request is admitted as soon as a
//     lane and its state's block are free; requests that arrive while others
//     are running are admitted at once if they fit, so their kernels overlap
//     on the device with the running ones (continuous batching).  Large
//     requests (>= large_qubits) may hold only `large_lanes` lanes at a time;
//     small requests run on high-priority streams, so their CTAs are scheduled
//     ahead of a large request's pass tiles whenever SM resources free up.
//   * Admission is first-come first-served with bounded bypass: a request that
//     does not fit yet may be overtaken by later ones that do, at most
//     kMaxBypass times, after which nothing behind it is admitted until it is.
//   * Each request's device work is the same sequence of launches (tiled
//     passes, FP64 reductions or sampling) with the same launch shapes as the
//     state API uses, on its own stream and scratch, so its result does not
//     depend on what else is running.
// Planning (lowering + tiled-pass plan) runs in submit(), on the caller's
// thread; the latency clock starts before it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "kernels.h"
#include "planner.h"
#include "tcrun.h"

namespace nqpu {
namespace {

constexpr uint32_t kMaxBypass = 64;
constexpr size_t kTableAlign = 256;

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Buddy allocator over `blocks` top-level blocks of 2^top bytes; every block
// handed out is 2^order bytes, order in [min, top].
class Buddy {
 public:
  void init(int min_order, int top_order, uint64_t blocks) {
    min_ = min_order;
    top_ = top_order;
    free_.assign(size_t(top_ - min_ + 1), {});
    for (uint64_t b = 0; b < blocks; ++b) free_[size_t(top_ - min_)].insert(b << top_);
    used_ = 0;
  }
  bool alloc(int order, uint64_t* off) {
    order = std::max(order, min_);
    if (order > top_) return false;
    int o = order;
    while (o <= top_ && free_[size_t(o - min_)].empty()) ++o;
    if (o > top_) return false;
    auto& fl = free_[size_t(o - min_)];
    uint64_t a = *fl.begin();  // lowest address first
    fl.erase(fl.begin());
    while (o > order) {
      --o;
      free_[size_t(o - min_)].insert(a + (1ull << o));
    }
    *off = a;
    used_ += 1ull << order;
    return true;
  }
  void release(uint64_t off, int order) {
    order = std::max(order, min_);
    used_ -= 1ull << order;
    while (order < top_) {
      const uint64_t buddy = off ^ (1ull << order);
      auto& fl = free_[size_t(order - min_)];
      auto it = fl.find(buddy);
      if (it == fl.end()) break;
      fl.erase(it);
      off = std::min(off, buddy);
      ++order;
    }
    free_[size_t(order - min_)].insert(off);
  }
  uint64_t used() const { return used_; }

 private:
  int min_ = 12, top_ = 12;
  std::vector<std::set<uint64_t>> free_;
  uint64_t used_ = 0;
};

struct Request {
  uint64_t id = 0;
  uint32_t n = 0;
  int kind = 0;
  uint32_t shots = 0;
  uint64_t seed = 0;
  bool tiled = false;
  TilePlan plan;
  bool tensor = false;                 // tensor-core passes (NQPU_MODE_AUTO's choice)
  TcPlan tcplan;
  std::vector<size_t> bmat_off;        // B operands of each pass, in halves after off_stages
  std::vector<Op> ops;                 // per-gate path (states below the tiled minimum)
  std::vector<unsigned char> tables;   // passes | stages | ops, kTableAlign-aligned parts
  size_t off_stages = 0, off_ops = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  std::vector<double> z;
  std::vector<uint64_t> outcomes;
  int status = 0;  // 0 queued, 1 running, 2 done, 3 failed
  NqpuError err = NQPU_OK;
  uint64_t mem_off = 0;
  int mem_order = 0;
  uint32_t bypassed = 0;
  bool large = false;
};

struct Lane {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool high = true;
  double* scratch = nullptr;
  double* d_small = nullptr;
  double* h_small = nullptr;
  double* d_uni = nullptr;
  double* h_uni = nullptr;
  uint64_t* d_shots = nullptr;
  uint64_t* h_shots = nullptr;
  unsigned char* d_tab = nullptr;
  unsigned char* h_tab = nullptr;
  size_t tab_cap = 0;
  double* d_tcnorm = nullptr;  // tensor passes: 3 x SM-count norm partials
  int* d_tcerr = nullptr;      // tensor passes: bounded-wait expiry flag
  int* h_tcerr = nullptr;
  std::vector<unsigned char*> old_h_tab;  // freed at shutdown
  std::shared_ptr<Request> req;
};

size_t align_up(size_t x) { return (x + kTableAlign - 1) / kTableAlign * kTableAlign; }

// Uniforms of the reference C FFI's xorshift64* stream for one seed (the same
// generator, seeding and [0,1) mapping as nqpu_set_seed + nqpu_sample).
void seeded_uniforms(uint64_t seed, double* out, uint32_t count) {
  uint64_t s = seed == 0 ? 0x853c49e6748fea9bull : seed;
  for (uint32_t i = 0; i < count; ++i) {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    const uint64_t v = s * 0x2545F4914F6CDD1Dull;
    out[i] = double(v >> 11) / double(1ull << 53);
  }
}

}  // namespace

struct ServerImpl {
  NqpuServerConfig cfg{};
  int device = 0;
  int sms = 148;
  char* d_arena = nullptr;
  uint64_t arena_bytes = 0;
  Buddy buddy;
  std::vector<Lane> lanes;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  std::thread worker;
  bool stop = false;
  uint64_t next_id = 1;
  uint64_t submitted = 0, completed = 0, failed = 0, running = 0, large_running = 0, cancelled = 0;
  uint64_t peak_used = 0, peak_running = 0;
};

namespace {

cudaError_t launch_request(ServerImpl* sv, Lane& L, Request& r) {
  cudaStream_t st = L.stream;
  cudaError_t e;
  void* amp = sv->d_arena + r.mem_off;
  if (r.tiled || r.tensor) {
    const size_t bytes = r.tables.size();
    if (bytes > L.tab_cap) {
      // grow the lane's table buffers: stream-ordered device free/alloc; the
      // old pinned buffer may still back a finished copy, keep it until exit
      if (L.d_tab && (e = cudaFreeAsync(L.d_tab, st)) != cudaSuccess) return e;
      L.d_tab = nullptr;
      if (L.h_tab) L.old_h_tab.push_back(L.h_tab);
      L.h_tab = nullptr;
      L.tab_cap = 0;
      const size_t cap = std::max<size_t>(bytes * 2, 1 << 20);
      if ((e = cudaMallocAsync(reinterpret_cast<void**>(&L.d_tab), cap, st)) != cudaSuccess) return e;
      if ((e = cudaMallocHost(reinterpret_cast<void**>(&L.h_tab), cap)) != cudaSuccess) return e;
      L.tab_cap = cap;
    }
    std::memcpy(L.h_tab, r.tables.data(), bytes);
    if ((e = cudaMemcpyAsync(L.d_tab, L.h_tab, bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  }
  if ((e = launch_set_basis(DType::C64, amp, int(r.n), 0, st, sv->sms)) != cudaSuccess) return e;
  if (r.tensor) {
    if ((e = cudaMemsetAsync(L.d_tcerr, 0, sizeof(int), st)) != cudaSuccess) return e;
    if ((e = tc_launch(static_cast<float*>(amp), r.tcplan, reinterpret_cast<const TcPassRec*>(L.d_tab),
                       reinterpret_cast<const uint16_t*>(L.d_tab + r.off_stages), r.bmat_off.data(), L.d_tcnorm,
                       sv->sms, L.d_tcerr, st)) != cudaSuccess)
      return e;
    if ((e = cudaMemcpyAsync(L.h_tcerr, L.d_tcerr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return e;
  } else if (r.tiled) {
    const PassRec* dp = reinterpret_cast<const PassRec*>(L.d_tab);
    const StageRec* ds = reinterpret_cast<const StageRec*>(L.d_tab + r.off_stages);
    const void* dops = L.d_tab + r.off_ops;
    for (size_t i = 0; i < r.plan.passes.size(); ++i)
      if ((e = launch_tile_pass(DType::C64, amp, int(r.n), r.plan.passes[i], dp, ds, dops, int(i), st,
                                sv->sms)) != cudaSuccess)
        return e;
  } else {
    for (const Op& op : r.ops)
      if ((e = launch_pergate(DType::C64, amp, int(r.n), op, st, sv->sms)) != cudaSuccess) return e;
  }
  if (r.kind == NQPU_REQUEST_ZALL) {
    if ((e = launch_zsums(DType::C64, amp, int(r.n), L.scratch, L.d_small, st, sv->sms)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(L.h_small, L.d_small, sizeof(double) * (r.n + 1), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      return e;
  } else {
    seeded_uniforms(r.seed, L.h_uni, r.shots);
    if ((e = cudaMemcpyAsync(L.d_uni, L.h_uni, sizeof(double) * r.shots, cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return e;
    if ((e = launch_sample(DType::C64, amp, int(r.n), L.d_uni, r.shots, L.scratch, L.d_shots, st, sv->sms)) !=
        cudaSuccess)
      return e;
    if ((e = cudaMemcpyAsync(L.h_shots, L.d_shots, sizeof(uint64_t) * r.shots, cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      return e;
  }
  return cudaEventRecord(L.done, st);
}

void finish(ServerImpl* sv, Lane& L, cudaError_t result) {
  std::shared_ptr<Request> r = std::move(L.req);
  L.req.reset();
  if (result == cudaSuccess && r->tensor && *L.h_tcerr) result = cudaErrorLaunchTimeout;  // a bounded wait expired
  if (result == cudaSuccess) {
    if (r->kind == NQPU_REQUEST_ZALL) {
      r->z.resize(r->n);
      for (uint32_t q = 0; q < r->n; ++q) r->z[q] = L.h_small[0] - 2.0 * L.h_small[1 + q];
    } else {
      r->outcomes.assign(L.h_shots, L.h_shots + r->shots);
    }
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  r->t_done = now_s();
  r->status = result == cudaSuccess ? 2 : 3;
  r->err = result == cudaSuccess ? NQPU_OK : NQPU_SIMULATION_FAILED;
  sv->buddy.release(r->mem_off, r->mem_order);
  sv->running--;
  if (r->large) sv->large_running--;
  if (result == cudaSuccess) sv->completed++;
  else sv->failed++;
  sv->cv_done.notify_all();
}

void worker_main(ServerImpl* sv) {
  cudaSetDevice(sv->device);
  std::vector<std::pair<size_t, std::shared_ptr<Request>>> to_launch;
  for (;;) {
    bool progressed = false;
    // completions
    for (Lane& L : sv->lanes) {
      if (!L.req) continue;
      const cudaError_t q = cudaEventQuery(L.done);
      if (q == cudaErrorNotReady) continue;
      finish(sv, L, q);
      progressed = true;
    }
    // admissions
    to_launch.clear();
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      if (sv->stop && sv->running == 0) break;
      Request* waiting = nullptr;  // oldest queued request that could not be admitted
      for (auto it = sv->pending.begin(); it != sv->pending.end();) {
        if (sv->running >= sv->lanes.size()) break;  // every lane busy
        Request& r = **it;
        // lane: large requests only on the low-priority lanes (at most
        // large_lanes of them), small ones on a high-priority lane if one is
        // free, else on a free low-priority lane
        size_t lane = sv->lanes.size();
        if (!r.large || sv->large_running < sv->cfg.large_lanes)
          for (size_t i = 0; i < sv->lanes.size(); ++i) {
            const Lane& L = sv->lanes[i];
            if (L.req) continue;
            if (r.large && L.high) continue;
            if (L.high == !r.large) {
              lane = i;
              break;
            }
            if (lane == sv->lanes.size()) lane = i;
          }
        uint64_t off = 0;
        if (lane < sv->lanes.size() && sv->buddy.alloc(int(r.n) + 3, &off)) {
          r.mem_off = off;
          r.mem_order = int(r.n) + 3;
          r.status = 1;
          r.t_admit = now_s();
          sv->running++;
          if (r.large) sv->large_running++;
          sv->peak_used = std::max(sv->peak_used, sv->buddy.used());
          sv->peak_running = std::max(sv->peak_running, sv->running);
          sv->lanes[lane].req = *it;
          to_launch.emplace_back(lane, *it);
          if (waiting) waiting->bypassed++;  // overtook an older request
          it = sv->pending.erase(it);
          continue;
        }
        // does not fit yet; later requests may overtake it, a bounded number of times
        if (!waiting) waiting = &r;
        if (waiting->bypassed >= kMaxBypass) break;
        ++it;
      }
      if (to_launch.empty() && !progressed) {
        if (sv->running == 0 && sv->pending.empty() && !sv->stop) {
          sv->cv_work.wait(lk);
        } else {
          sv->cv_work.wait_for(lk, std::chrono::microseconds(20));
        }
        continue;
      }
    }
    for (auto& p : to_launch) {
      Lane& L = sv->lanes[p.first];
      const cudaError_t e = launch_request(sv, L, *p.second);
      if (e != cudaSuccess) {
        cudaStreamSynchronize(L.stream);
        cudaGetLastError();
        finish(sv, L, e);
      }
    }
  }
}

void server_free(ServerImpl* sv) {
  for (Lane& L : sv->lanes) {
    if (L.stream) cudaStreamSynchronize(L.stream);
    if (L.d_tab) cudaFreeAsync(L.d_tab, L.stream);
    if (L.stream) cudaStreamSynchronize(L.stream);
    if (L.done) cudaEventDestroy(L.done);
    if (L.scratch) cudaFree(L.scratch);
    if (L.d_small) cudaFree(L.d_small);
    if (L.d_uni) cudaFree(L.d_uni);
    if (L.d_shots) cudaFree(L.d_shots);
    if (L.h_small) cudaFreeHost(L.h_small);
    if (L.h_uni) cudaFreeHost(L.h_uni);
    if (L.h_shots) cudaFreeHost(L.h_shots);
    if (L.d_tcnorm) cudaFree(L.d_tcnorm);
    if (L.d_tcerr) cudaFree(L.d_tcerr);
    if (L.h_tcerr) cudaFreeHost(L.h_tcerr);
    if (L.h_tab) cudaFreeHost(L.h_tab);
    for (unsigned char* p : L.old_h_tab) cudaFreeHost(p);
    if (L.stream) cudaStreamDestroy(L.stream);
  }
  if (sv->d_arena) cudaFree(sv->d_arena);
  delete sv;
}

}  // namespace
}  // namespace nqpu

using namespace nqpu;

static ServerImpl* SV(NqpuServer* h) { return reinterpret_cast<ServerImpl*>(h); }

extern "C" NqpuServer* nqpu_server_create(const NqpuServerConfig* config) {
  if (!device_ready()) return nullptr;
  NqpuServerConfig c{};
  if (config) c = *config;
  if (c.max_qubits == 0) c.max_qubits = 28;
  if (c.lanes == 0) c.lanes = 16;
  if (c.large_lanes == 0) c.large_lanes = 2;
  if (c.large_qubits == 0) c.large_qubits = 22;
  if (c.max_shots == 0) c.max_shots = 1024;
  if (c.max_qubits > 32 || c.lanes > 64 || c.large_lanes > c.lanes || c.max_shots > (1u << 24)) return nullptr;
  const uint64_t top = 1ull << (c.max_qubits + 3);  // largest state, complex64
  if (c.hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return nullptr;
    c.hbm_budget_bytes = uint64_t(fr) / 2;
  }
  const uint64_t blocks = c.hbm_budget_bytes / top;
  if (blocks == 0) return nullptr;  // the budget must hold one largest state
  auto* sv = new (std::nothrow) ServerImpl();
  if (!sv) return nullptr;
  sv->cfg = c;
  cudaGetDevice(&sv->device);
  sv->sms = device_sms();
  sv->arena_bytes = blocks * top;
  bool ok = cudaMalloc(reinterpret_cast<void**>(&sv->d_arena), sv->arena_bytes) == cudaSuccess;
  sv->buddy.init(12, int(c.max_qubits) + 3, blocks);
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  sv->lanes.resize(c.lanes);
  const size_t scratch = reduce_scratch_bytes(int(c.max_qubits));
  for (uint32_t i = 0; ok && i < c.lanes; ++i) {
    Lane& L = sv->lanes[i];
    L.high = i >= c.large_lanes;  // the first large_lanes lanes are the low-priority ones
    ok = ok && cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, L.high ? prio_high : prio_low) ==
                   cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.scratch), scratch) == cudaSuccess;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.d_small), 64 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMallocHost(reinterpret_cast<void**>(&L.h_small), 64 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.d_uni), c.max_shots * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMallocHost(reinterpret_cast<void**>(&L.h_uni), c.max_shots * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.d_shots), c.max_shots * sizeof(uint64_t)) == cudaSuccess;
    ok = ok && cudaMallocHost(reinterpret_cast<void**>(&L.h_shots), c.max_shots * sizeof(uint64_t)) == cudaSuccess;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.d_tcnorm), 3 * size_t(sv->sms) * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(reinterpret_cast<void**>(&L.d_tcerr), sizeof(int)) == cudaSuccess;
    ok = ok && cudaMallocHost(reinterpret_cast<void**>(&L.h_tcerr), sizeof(int)) == cudaSuccess;
    if (ok) *L.h_tcerr = 0;
  }
  if (!ok) {
    cudaGetLastError();
    server_free(sv);
    return nullptr;
  }
  sv->worker = std::thread(worker_main, sv);
  return reinterpret_cast<NqpuServer*>(sv);
}

extern "C" void nqpu_server_destroy(NqpuServer* server) {
  if (!server) return;
  ServerImpl* sv = SV(server);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    sv->pending.clear();  // queued requests are dropped; running ones finish
  }
  sv->cv_work.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  server_free(sv);
}

extern "C" NqpuError nqpu_server_submit(NqpuServer* server, const NqpuCircuit* circuit, NqpuRequestKind kind,
                                        uint32_t shots, uint64_t seed, uint64_t* request_id) {
  if (!server || !circuit || !request_id) return NQPU_NULL_POINTER;
  ServerImpl* sv = SV(server);
  const double t0 = now_s();
  const CircuitImpl* c = reinterpret_cast<const CircuitImpl*>(circuit);
  if (c->n == 0 || c->n > sv->cfg.max_qubits) return NQPU_INVALID_PARAMETER;
  if (circuit_has_mid(c->gates)) return NQPU_INVALID_PARAMETER;  // measurement-free circuits only
  if (kind != NQPU_REQUEST_ZALL && kind != NQPU_REQUEST_SHOTS) return NQPU_INVALID_PARAMETER;
  if (kind == NQPU_REQUEST_SHOTS && (shots == 0 || shots > sv->cfg.max_shots)) return NQPU_INVALID_PARAMETER;
  auto r = std::make_shared<Request>();
  r->t_submit = t0;
  r->n = c->n;
  r->kind = int(kind);
  r->shots = kind == NQPU_REQUEST_SHOTS ? shots : 0;
  r->seed = seed;
  r->large = c->n >= sv->cfg.large_qubits;
  std::vector<Op> ops = lower_circuit(c->gates);
  if (auto_mode_for(ops, c->n, DType::C64) == NQPU_MODE_TENSOR) {
    // the engine's own choice (NQPU_MODE_AUTO): tensor-core passes; tables =
    // pass records | B operands
    std::string err;
    if (!build_tc_plan(ops, int(c->n), &r->tcplan, &err)) return NQPU_INVALID_PARAMETER;
    r->tensor = true;
    tc_bmat_offsets(r->tcplan, &r->bmat_off);
    const size_t bp = r->tcplan.passes.size() * sizeof(TcPassRec);
    const size_t bb = r->tcplan.bmats.size() * sizeof(uint16_t);
    r->off_stages = align_up(bp);
    r->tables.assign(r->off_stages + std::max<size_t>(bb, 1), 0);
    if (bp) std::memcpy(r->tables.data(), r->tcplan.passes.data(), bp);
    if (bb) std::memcpy(r->tables.data() + r->off_stages, r->tcplan.bmats.data(), bb);
    r->tcplan.unitaries.clear();  // FP64 copies for tests only
    r->tcplan.bmats.clear();
    r->tcplan.bmats.shrink_to_fit();
  } else if (int(c->n) >= tile_min_qubits(DType::C64)) {
    std::string err;
    if (!build_tile_plan(ops, int(c->n), DType::C64, tile_kmax_for(DType::C64), &r->plan, &err))
      return NQPU_INVALID_PARAMETER;
    r->tiled = true;
    const TilePlan& p = r->plan;
    const size_t bp = p.passes.size() * sizeof(PassRec);
    const size_t bs = p.stages.size() * sizeof(StageRec);
    const size_t bo = p.ops_f.size() * sizeof(TileOp<float>);
    r->off_stages = align_up(bp);
    r->off_ops = r->off_stages + align_up(bs);
    r->tables.assign(r->off_ops + std::max<size_t>(bo, 1), 0);
    if (bp) std::memcpy(r->tables.data(), p.passes.data(), bp);
    if (bs) std::memcpy(r->tables.data() + r->off_stages, p.stages.data(), bs);
    if (bo) std::memcpy(r->tables.data() + r->off_ops, p.ops_f.data(), bo);
  } else {
    r->ops = std::move(ops);
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return NQPU_INVALID_HANDLE;
    r->id = sv->next_id++;
    sv->reqs[r->id] = r;
    sv->pending.push_back(r);
    sv->submitted++;
    *request_id = r->id;
  }
  sv->cv_work.notify_one();
  return NQPU_OK;
}

extern "C" NqpuError nqpu_server_poll(NqpuServer* server, uint64_t request_id, int32_t* done) {
  if (!server || !done) return NQPU_NULL_POINTER;
  ServerImpl* sv = SV(server);
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(request_id);
  if (it == sv->reqs.end()) return NQPU_INVALID_HANDLE;
  *done = it->second->status >= 2 ? 1 : 0;
  return NQPU_OK;
}

extern "C" NqpuError nqpu_server_wait(NqpuServer* server, uint64_t request_id, double timeout_s) {
  if (!server) return NQPU_NULL_POINTER;
  ServerImpl* sv = SV(server);
  std::unique_lock<std::mutex> lk(sv->mu);
  auto ready = [&]() {
    if (request_id == 0) return sv->pending.empty() && sv->running == 0;
    auto it = sv->reqs.find(request_id);
    return it == sv->reqs.end() || it->second->status >= 2;
  };
  if (request_id != 0 && sv->reqs.find(request_id) == sv->reqs.end()) return NQPU_INVALID_HANDLE;
  const auto limit = std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 3600.0);
  if (!sv->cv_done.wait_for(lk, limit, ready)) return NQPU_SIMULATION_FAILED;  // timed out
  return NQPU_OK;
}

extern "C" NqpuError nqpu_server_result(NqpuServer* server, uint64_t request_id, double* out_z, uint32_t z_len,
                                        uint64_t* out_shots, uint32_t shots_len, double* timing_ms) {
  if (!server) return NQPU_NULL_POINTER;
  ServerImpl* sv = SV(server);
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(request_id);
  if (it == sv->reqs.end()) return NQPU_INVALID_HANDLE;
  const Request& r = *it->second;
  if (r.status < 2) return NQPU_INVALID_PARAMETER;  // not finished
  if (r.status == 3) {
    const NqpuError e = r.err;
    sv->reqs.erase(it);
    return e;
  }
  if (r.kind == NQPU_REQUEST_ZALL) {
    if (!out_z) return NQPU_NULL_POINTER;
    if (z_len < r.n) return NQPU_INVALID_PARAMETER;
    std::memcpy(out_z, r.z.data(), sizeof(double) * r.n);
  } else {
    if (!out_shots) return NQPU_NULL_POINTER;
    if (shots_len < r.shots) return NQPU_INVALID_PARAMETER;
    std::memcpy(out_shots, r.outcomes.data(), sizeof(uint64_t) * r.shots);
  }
  if (timing_ms) {
    timing_ms[0] = 1e3 * (r.t_admit - r.t_submit);
    timing_ms[1] = 1e3 * (r.t_done - r.t_admit);
    timing_ms[2] = 1e3 * (r.t_done - r.t_submit);
  }
  sv->reqs.erase(it);
  return NQPU_OK;
}

extern "C" NqpuError nqpu_server_cancel(NqpuServer* server, uint64_t request_id) {
  if (!server) return NQPU_NULL_POINTER;
  ServerImpl* sv = SV(server);
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(request_id);
  if (it == sv->reqs.end()) return NQPU_INVALID_HANDLE;
  // status is set to running under this lock when the worker admits a request,
  // so a request still queued here is still in `pending`
  if (it->second->status != 0) return NQPU_INVALID_PARAMETER;  // admitted: it runs to completion
  auto pit = std::find(sv->pending.begin(), sv->pending.end(), it->second);
  if (pit != sv->pending.end()) sv->pending.erase(pit);
  sv->reqs.erase(it);
  sv->cancelled++;
  sv->cv_done.notify_all();  // wait(0) may now be satisfied
  return NQPU_OK;
}

extern "C" NqpuError nqpu_server_stats(NqpuServer* server, uint64_t* out, uint32_t len) {
  if (!server || !out) return NQPU_NULL_POINTER;
  if (len < 8) return NQPU_INVALID_PARAMETER;
  ServerImpl* sv = SV(server);
  std::lock_guard<std::mutex> lk(sv->mu);
  out[0] = sv->submitted;
  out[1] = sv->completed;
  out[2] = sv->failed;
  out[3] = sv->running;
  out[4] = sv->pending.size();
  out[5] = sv->peak_used;
  out[6] = sv->arena_bytes;
  out[7] = sv->peak_running;
  if (len >= 9) out[8] = sv->cancelled;
  return NQPU_OK;
}
