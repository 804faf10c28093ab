// server.cu -- the serving loop: sampling requests submitted at any time, kept
// resident on the device and run with continuous batching.
//
// A request is a circuit (op list), a shot count and a seed.  Its program is
// compiled once per distinct op list and stays resident (a cache keyed by
// the op bytes, compared in full on a hash hit; programs count against the
// HBM budget, and unused ones are evicted least recently used first when it
// runs short).  Admission is first come, first served against an HBM
// budget, a number of slots and the GPU's fill: the head of the queue is
// admitted as soon as a slot is free, its memory (the full record, plus one
// chunk's frame planes) fits the budget and the running requests' remaining
// walker CTAs leave SMs idle (a request with two or more chunks to go fills
// the GPU; one on its last chunk leaves the SMs that chunk does not use).  Device memory comes from the stream-ordered
// allocator (cudaMallocAsync / cudaFreeAsync on the slot's stream), so the
// scheduler thread never waits for the device.  An admitted request runs on its
// slot's stream as a sequence of shot chunks (fresh Philox runs with the
// chunk's global shot offset, each writing its columns of the request's
// record; every record equals that of one plain run of the request), two
// chunks in flight at a time.  So the oldest requests keep the SMs they fill
// (first come, first served, as serial execution, which bounds the longest
// waits) and later ones run beside them only on SMs they leave idle: small
// requests, and the last chunk of a large one.  A scheduler thread admits,
// launches chunks and retires (CUDA events); the caller polls, waits, copies
// results out and releases them.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "qcb_internal.h"

namespace qcb {

enum ReqState : int32_t { RQ_QUEUED = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = 3 };

// A resident compiled program: its op list (compared byte for byte on a hash
// hit), its device bytes (charged to the budget), the requests holding it.
struct CachedProgram {
  std::vector<qcb_op> ops;
  qcb_program* prog = nullptr;
  uint64_t hash = 0, bytes = 0, refs = 0, last_use = 0;
};

struct Request {
  uint64_t id = 0;
  std::vector<qcb_op> ops;
  uint64_t shots = 0, seed = 0;
  qcb_program* prog = nullptr;  // cached, owned by the server
  CachedProgram* cached = nullptr;
  uint64_t nbits = 0, ncols = 0, rec_pitch = 0;
  uint64_t bytes = 0;           // record + chunk planes charged to the budget
  uint32_t* record = nullptr;
  qcb_frame* chunk[2] = {nullptr, nullptr};  // chunk frames: chunk k runs in chunk[k & 1] (one for a one-chunk request)
  int slot = -1;
  cudaStream_t stream[2] = {nullptr, nullptr};  // the slot's streams: chunk k runs on stream[k & 1]
  uint64_t chunk_w = 0;                              // columns per chunk (whole walker waves)
  uint64_t chunk_bytes = 0;                          // chunk frames: planes + noise pre-sampler scratch
  uint64_t nchunks = 0, launched = 0, finished = 0;  // chunks: total, launched, seen complete
  uint32_t ctas_full = 0, ctas_last = 0;             // walker CTAs of a full and of the last chunk
  cudaEvent_t chunk_ev[2] = {nullptr, nullptr};      // completion of chunk k in chunk_ev[k % 2]
  cudaEvent_t done = nullptr;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int32_t state = RQ_QUEUED;
  int32_t status = QCB_OK;
  std::string msg;  // the error message of a failed request
};

// The calling thread's last error message (errors are per thread).
static std::string last_msg() {
  char buf[512];
  qcb_last_error(buf, sizeof(buf));
  return std::string(buf);
}

}  // namespace qcb

struct qcb_server {
  int device = 0;
  uint64_t budget = 0, used = 0;
  uint32_t nslots = 0;
  uint64_t chunk_cols = 0;  // columns per chunk (a multiple of 32: 1024-shot groups)
  std::vector<cudaStream_t> streams;  // two per slot (slot k: 2k, 2k + 1)
  bool fill_gate = true;              // admit only onto idle SMs (false: whenever a slot is free)
  uint32_t capacity = 0;              // walker CTAs the GPU runs at once (one per SM)
  std::vector<int64_t> slot_req;  // request id per slot, -1 when free
  std::map<uint64_t, std::unique_ptr<qcb::Request>> reqs;
  std::deque<uint64_t> queue;
  std::deque<uint64_t> completed;  // finished or failed, not yet reported by next_done
  std::unordered_multimap<uint64_t, std::unique_ptr<qcb::CachedProgram>> programs;
  uint64_t program_bytes = 0;  // device bytes of the resident programs (inside `used`)
  uint64_t use_clock = 0;
  int32_t* slot_status = nullptr;  // pinned: each slot's last walker status word
  uint64_t next_id = 1;
  std::mutex mu;
  std::condition_variable cv;   // wakes the scheduler
  std::condition_variable done_cv;
  std::thread th;
  bool stop = false;
  std::chrono::steady_clock::time_point t0;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace qcb {

// Admission policy knob: 1 (default) admits a request only while the running
// ones leave SMs idle, 0 whenever a slot is free (the GPU's block scheduler
// then interleaves the requests' chunks).
static uint32_t g_server_fill = 1;
void set_server_fill(uint32_t v) { g_server_fill = v; }

// Test knob: keep only this many low bits of the program hash (0: all 64),
// so that distinct circuits collide and the byte comparison decides.
static uint32_t g_hash_bits = 0;
void set_server_hash_bits(uint32_t b) { g_hash_bits = b; }

static uint64_t ops_hash(const std::vector<qcb_op>& ops) {
  uint64_t h = 1469598103934665603ull;
  const uint8_t* p = (const uint8_t*)ops.data();
  for (size_t i = 0; i < ops.size() * sizeof(qcb_op); i++) { h ^= p[i]; h *= 1099511628211ull; }
  h ^= ops.size() * 0x9E3779B97F4A7C15ull;
  return (g_hash_bits && g_hash_bits < 64) ? (h & ((1ull << g_hash_bits) - 1)) : h;
}

// Device bytes of a compiled program (what it holds resident).
static uint64_t program_footprint(const qcb_program* p) {
  return p->stream_slot.size() * 4 + p->classes.size() * sizeof(NoiseClass) + p->cdf.size() * 4 +
         p->slot_qubit.size() * 4 + (uint64_t)p->qubit_slot_len * 4 + p->slot_swap.size() * 4 + 6 * 16;
}

// The resident program with exactly these ops, or null (lock held).
static CachedProgram* find_program(qcb_server* s, uint64_t h, const std::vector<qcb_op>& ops) {
  auto range = s->programs.equal_range(h);
  for (auto it = range.first; it != range.second; ++it) {
    CachedProgram* c = it->second.get();
    if (c->ops.size() == ops.size() &&
        (ops.empty() || std::memcmp(c->ops.data(), ops.data(), ops.size() * sizeof(qcb_op)) == 0))
      return c;
  }
  return nullptr;
}

// Evict unused programs, least recently used first, until `need` more bytes
// fit the budget (lock held).  Returns whether they fit.
static bool evict_programs(qcb_server* s, uint64_t need) {
  while (s->used + need > s->budget) {
    auto victim = s->programs.end();
    for (auto it = s->programs.begin(); it != s->programs.end(); ++it)
      if (!it->second->refs && (victim == s->programs.end() || it->second->last_use < victim->second->last_use))
        victim = it;
    if (victim == s->programs.end()) return false;
    s->used -= victim->second->bytes;
    s->program_bytes -= victim->second->bytes;
    qcb_program_destroy(victim->second->prog);  // no request holds it: no work of it is in flight
    s->programs.erase(victim);
  }
  return true;
}

// Insert a freshly compiled program (lock held) unless an equal one arrived
// meanwhile; returns the resident one.  Its bytes are charged to the budget,
// evicting unused programs to make room where possible.
static CachedProgram* insert_program(qcb_server* s, uint64_t h, std::vector<qcb_op>&& ops, qcb_program* p) {
  if (CachedProgram* c = find_program(s, h, ops)) {
    qcb_program_destroy(p);
    return c;
  }
  auto c = std::make_unique<CachedProgram>();
  c->ops = std::move(ops);
  c->prog = p;
  c->hash = h;
  c->bytes = program_footprint(p);
  evict_programs(s, c->bytes);
  s->used += c->bytes;
  s->program_bytes += c->bytes;
  CachedProgram* raw = c.get();
  s->programs.emplace(h, std::move(c));
  return raw;
}

static uint64_t chunk_plane_bytes(uint32_t nq1, uint64_t chunk_cols) {
  const uint64_t pitch = std::max<uint64_t>(32, (chunk_cols + 31) / 32 * 32);
  return (uint64_t)2 * (nq1 + 1) * pitch * 4 + (uint64_t)pitch * 4 + 16;
}

// Walker CTAs still to run for a running request: a full chunk's while two or
// more chunks remain (it fills the GPU as serial execution would), the last
// chunk's while only that one remains, 0 once every chunk has finished.
static uint64_t remaining_ctas(const Request& r) {
  const uint64_t left = r.nchunks - r.finished;
  return left >= 2 ? r.ctas_full : left == 1 ? r.ctas_last : 0;
}

// Free a chunk frame's device buffers in stream order (the status word is
// shared by the two frames and freed with the first).
static void free_chunk_frame(qcb_frame* cf, bool err, cudaStream_t st) {
  if (!cf) return;
  if (cf->planes) cudaFreeAsync(cf->planes, st);
  if (cf->pre) cudaFreeAsync(cf->pre, st);
  if (err && cf->err) cudaFreeAsync(cf->err, st);
  cf->planes = nullptr;
  cf->pre = nullptr;
  cf->pre_bytes = 0;
  cf->err = nullptr;
}

// After the last chunk: stream 0 joins stream 1, then the walker status word
// to the slot's pinned word, the chunk frames back to the pool and the
// request's completion event, all in stream order.
static int finish_launches(qcb_server* s, Request& r) {
  int status = r.status;
  if (r.chunk[1] && (cudaEventRecord(r.chunk_ev[1], r.stream[1]) != cudaSuccess ||
                     cudaStreamWaitEvent(r.stream[0], r.chunk_ev[1], 0) != cudaSuccess) && status == QCB_OK)
    status = fail(QCB_ECUDA, "serving: stream join");
  qcb_frame* cf = r.chunk[0];
  if (status == QCB_OK && cf->err &&
      cudaMemcpyAsync(&s->slot_status[r.slot], cf->err, 4, cudaMemcpyDeviceToHost, r.stream[0]) != cudaSuccess)
    status = fail(QCB_ECUDA, "serving: status copy");
  free_chunk_frame(r.chunk[1], false, r.stream[0]);
  free_chunk_frame(r.chunk[0], true, r.stream[0]);
  if (cudaEventRecord(r.done, r.stream[0]) != cudaSuccess && status == QCB_OK)
    status = fail(QCB_ECUDA, "serving: event");
  return status;
}

// Launch the request's next chunk (lock held): chunk k in frame k & 1 on
// stream k & 1, so that consecutive chunks overlap (the next one's CTAs take
// the SMs the last wave of this one leaves, instead of one tail per chunk);
// after the last one, finish_launches.  A failure ends the launches: the
// request retires as failed once its streams have drained.
static void launch_chunk(qcb_server* s, Request& r) {
  const uint64_t k = r.launched;
  const uint32_t j = r.chunk[1] ? (uint32_t)(k & 1) : 0u;
  const uint64_t c0 = k * r.chunk_w;
  const uint64_t nc = std::min<uint64_t>(r.chunk_w, r.ncols - c0);
  int status = run_chunk(r.chunk[j], nc, r.prog, r.seed, c0 * 32, r.record + c0, r.rec_pitch, r.stream[j]);
  if (status == QCB_OK && cudaEventRecord(r.chunk_ev[k % 2], r.stream[j]) != cudaSuccess)
    status = fail(QCB_ECUDA, "serving: chunk event");
  r.launched++;
  if (status != QCB_OK) {
    r.status = status;
    r.msg = last_msg();
    r.launched = r.nchunks;  // no further chunks
  }
  if (r.launched == r.nchunks) {
    const int st = finish_launches(s, r);
    if (st != QCB_OK && r.status == QCB_OK) {
      r.status = st;
      r.msg = last_msg();
    }
  }
}

// Keep two chunks of every running request in flight (lock held): count the
// chunks seen complete and launch the next while fewer than two are pending.
static void advance(qcb_server* s) {
  for (uint32_t k = 0; k < s->nslots; k++) {
    if (s->slot_req[k] < 0) continue;
    Request& r = *s->reqs[(uint64_t)s->slot_req[k]];
    while (r.finished < r.launched && r.status == QCB_OK) {
      if (cudaEventQuery(r.chunk_ev[r.finished % 2]) != cudaSuccess) break;
      r.finished++;
    }
    while (r.launched < r.nchunks && r.launched - r.finished < 2) launch_chunk(s, r);
  }
}

// Noise pre-sampler scratch per chunk frame: chunks are narrowed (by whole
// waves) until their scratch fits this, so that strong noise is pre-sampled
// too (d = 11, 2^20 shots, p = 1e-2: 2.14 ms pre-sampled, 4.82 ms drawn in
// the walk).
constexpr uint64_t SERVE_PRESAMPLE_MAX = 1ull << 30;

// Pre-sampler scratch of a chunk frame of `cw` columns (0: drawn in the walk).
static uint64_t chunk_pre_bytes(const Request& r, uint64_t cw) {
  const uint64_t need = chunk_presample_bytes(r.prog, cw);
  return need <= SERVE_PRESAMPLE_MAX ? need : 0;
}

// Columns per chunk of a request: all of them (one launch) when they fit the
// server's chunk width, else the nearest whole number of walker waves (one
// tile per SM) to it that is a whole number of 1024-shot groups, so that no
// chunk but the last ends on a mostly empty wave; then fewer waves while the
// chunk's pre-sampler scratch does not fit SERVE_PRESAMPLE_MAX.
static uint64_t chunk_width(const qcb_server* s, const Request& r) {
  if (r.ncols <= s->chunk_cols) return r.ncols;  // one launch
  uint32_t T = 0;
  chunk_shape(r.prog, s->chunk_cols, &T, nullptr);
  uint64_t unit = (uint64_t)s->capacity * std::max<uint32_t>(T, 1);
  while (unit % 32) unit *= 2;
  const uint64_t k0 = std::max<uint64_t>(1, (s->chunk_cols + unit / 2) / unit);
  uint64_t cw = std::min(k0 * unit, r.ncols);
  if (chunk_presample_bytes(r.prog, cw) > SERVE_PRESAMPLE_MAX && cw > unit) {
    uint64_t k = cw / unit;
    while (k > 1 && chunk_presample_bytes(r.prog, k * unit) > SERVE_PRESAMPLE_MAX) k--;
    if (chunk_presample_bytes(r.prog, k * unit) <= SERVE_PRESAMPLE_MAX) cw = k * unit;
  }
  return cw;
}

// Admit the head of the queue while a slot, the budget and the GPU's fill
// allow (called with the lock held), launching the first two chunks of each
// admitted request on its slot's stream.
static void admit(qcb_server* s) {
  while (!s->queue.empty()) {
    int slot = -1;
    for (uint32_t k = 0; k < s->nslots; k++)
      if (s->slot_req[k] < 0) { slot = (int)k; break; }
    if (slot < 0) return;
    Request& r = *s->reqs[s->queue.front()];
    if (!r.bytes) {
      r.nbits = std::max<uint32_t>(r.prog->info.nbits, 1);
      r.ncols = (r.shots + 31) / 32;
      r.rec_pitch = std::max<uint64_t>(32, (r.ncols + 31) / 32 * 32);
      r.chunk_w = chunk_width(s, r);
      r.nchunks = (r.ncols + r.chunk_w - 1) / r.chunk_w;
      r.chunk_bytes = (r.nchunks > 1 ? 2 : 1) * (chunk_plane_bytes(std::max<uint32_t>(r.prog->nq, 1), r.chunk_w) +
                                                 chunk_pre_bytes(r, r.chunk_w));
      r.bytes = r.nbits * r.rec_pitch * 4 + r.chunk_bytes;
    }
    if (r.bytes > s->budget) {
      r.state = RQ_FAILED;
      r.status = QCB_EOOM;
      r.msg = "serving: the request needs more device memory than the server's budget";
      r.t_done = s->now();
      s->queue.pop_front();
      s->completed.push_back(r.id);
      s->done_cv.notify_all();
      continue;
    }
    bool running = false;
    uint64_t busy = 0;
    for (int64_t v : s->slot_req) {
      if (v < 0) continue;
      running = true;
      busy += remaining_ctas(*s->reqs[(uint64_t)v]);
    }
    // the SMs are taken (balanced tiles leave a wave a few CTAs short of the
    // SM count, so fewer than 1/16 idle counts as full): wait, in order
    if (s->fill_gate && running && busy + s->capacity / 16 > s->capacity) return;
    if (s->used + r.bytes > s->budget && !evict_programs(s, r.bytes)) {
      if (running) return;  // first come, first served: wait for memory
      // nothing runs and nothing more can be evicted: the resident programs
      // of queued requests leave no room for this one
      r.state = RQ_FAILED;
      r.status = QCB_EBUDGET;
      r.msg = "serving: the programs of queued requests leave too little of the budget for this request";
      r.t_done = s->now();
      s->queue.pop_front();
      s->completed.push_back(r.id);
      s->done_cv.notify_all();
      continue;
    }
    const uint32_t nq1 = std::max<uint32_t>(r.prog->nq, 1);
    cudaStream_t st = s->streams[2 * (size_t)slot];
    r.stream[0] = st;
    r.stream[1] = s->streams[2 * (size_t)slot + 1];
    r.slot = slot;
    r.launched = r.finished = 0;
    chunk_shape(r.prog, r.chunk_w, nullptr, &r.ctas_full);
    chunk_shape(r.prog, r.ncols - (r.nchunks - 1) * r.chunk_w, nullptr, &r.ctas_last);
    // the chunk frames (two when there are two or more chunks): planes for
    // one chunk and its noise pre-sampler scratch, allocated on stream 0 and
    // freed in stream order (no device-wide synchronisation on the
    // scheduler thread); one status word for both
    const uint64_t pre = chunk_pre_bytes(r, r.chunk_w);
    cudaError_t e = cudaSuccess;
    for (uint32_t f = 0; f < (r.nchunks > 1 ? 2u : 1u); f++) {
      qcb_frame* cf = new qcb_frame();
      cf->frames = r.chunk_w * 32;
      cf->qubits = nq1 - 1;
      cf->nq1 = nq1;
      cf->nbits = 0;
      cf->ncols = r.chunk_w;
      cf->pitch = std::max<uint64_t>(32, (r.chunk_w + 31) / 32 * 32);
      cf->planes = nullptr;
      cf->record = nullptr;
      cf->err = nullptr;
      r.chunk[f] = cf;
      if (e == cudaSuccess) e = cudaMallocAsync(&cf->planes, (size_t)2 * (nq1 + 1) * cf->pitch * 4, st);
      if (e == cudaSuccess && pre) {
        e = cudaMallocAsync(&cf->pre, pre, st);
        if (e == cudaSuccess) cf->pre_bytes = pre;
      }
    }
    if (e == cudaSuccess) e = cudaMallocAsync(&r.chunk[0]->err, 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r.chunk[0]->err, 0, 16, st);
    if (r.chunk[1]) r.chunk[1]->err = r.chunk[0]->err;
    if (e == cudaSuccess) e = cudaMallocAsync(&r.record, r.nbits * r.rec_pitch * 4, st);
    for (int k = 0; k < 2 && e == cudaSuccess; k++)
      if (!r.chunk_ev[k]) e = cudaEventCreateWithFlags(&r.chunk_ev[k], cudaEventDisableTiming);
    if (e == cudaSuccess && !r.done) e = cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming);
    // stream 1 starts after the allocations made on stream 0
    if (e == cudaSuccess && r.chunk[1]) e = cudaEventRecord(r.chunk_ev[1], st);
    if (e == cudaSuccess && r.chunk[1]) e = cudaStreamWaitEvent(r.stream[1], r.chunk_ev[1], 0);
    s->queue.pop_front();
    r.t_admit = s->now();
    if (e != cudaSuccess) {
      r.status = cuda_fail(e, "serving: admission");
      r.msg = last_msg();
      free_chunk_frame(r.chunk[1], false, st);
      free_chunk_frame(r.chunk[0], true, st);
      if (r.record) cudaFreeAsync(r.record, st);
      r.record = nullptr;
      for (qcb_frame*& cf : r.chunk) {
        delete cf;
        cf = nullptr;
      }
      r.slot = -1;
      r.state = RQ_FAILED; r.t_done = s->now();
      s->completed.push_back(r.id);
      s->done_cv.notify_all();
      continue;
    }
    r.state = RQ_RUNNING;
    s->slot_req[slot] = (int64_t)r.id;
    s->used += r.bytes;
    while (r.launched < r.nchunks && r.launched < 2) launch_chunk(s, r);
  }
}

// Retire the running requests whose launches have all been made and whose
// stream has drained (lock held): their chunk planes were freed in stream
// order, their records stay until released.
static void retire(qcb_server* s) {
  for (uint32_t k = 0; k < s->nslots; k++) {
    if (s->slot_req[k] < 0) continue;
    Request& r = *s->reqs[(uint64_t)s->slot_req[k]];
    if (r.launched < r.nchunks) continue;
    const cudaError_t q = cudaEventQuery(r.done);
    if (q == cudaErrorNotReady) continue;
    r.t_done = s->now();
    r.state = q == cudaSuccess && r.status == QCB_OK ? RQ_DONE : RQ_FAILED;
    if (q != cudaSuccess) {
      r.status = cuda_fail(q, "serving: request");
      r.msg = last_msg();
    }
    const int32_t h = *(volatile int32_t*)&s->slot_status[k];  // copied in stream order before the event
    if (r.state == RQ_DONE && h) {
      r.state = RQ_FAILED;
      r.status = h;
      r.msg = "serving: a device-side wait of the frame walker expired; the record is not valid";
    }
    s->slot_status[k] = 0;
    r.finished = r.nchunks;
    for (qcb_frame*& cf : r.chunk) {
      delete cf;
      cf = nullptr;
    }
    // the chunk planes leave the request's charge; the record stays charged
    s->used -= r.chunk_bytes;
    r.bytes -= r.chunk_bytes;
    s->slot_req[k] = -1;
    s->completed.push_back(r.id);
    s->done_cv.notify_all();
  }
}

static void scheduler(qcb_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    advance(s);
    retire(s);
    admit(s);
    bool running = false;
    for (int64_t v : s->slot_req) running |= v >= 0;
    // poll completions every 50 us while work is on the device, else sleep
    // until a submission
    if (running) s->cv.wait_for(lk, std::chrono::microseconds(50));
    else if (!s->stop) s->cv.wait(lk);  // a submission, a release or shutdown wakes it
  }
}

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_server_create(uint64_t hbm_budget_bytes, uint32_t slots, uint64_t chunk_shots, qcb_server** out) {
  if (!out) return fail(QCB_EARG, "null argument");
  *out = nullptr;
  if (!hbm_budget_bytes || !slots || slots > 64) return fail(QCB_EARG, "serving: budget > 0 and 1..64 slots");
  if (chunk_shots && chunk_shots % NOISE_GROUP) return fail(QCB_EARG, "serving: chunk_shots must be a multiple of 1024");
  auto s = std::make_unique<qcb_server>();
  QCB_CUDA(cudaGetDevice(&s->device));
  s->budget = hbm_budget_bytes;
  s->nslots = slots;
  s->chunk_cols = (chunk_shots ? chunk_shots : (uint64_t)1 << 20) / 32;
  s->slot_req.assign(slots, -1);
  QCB_CUDA(cudaHostAlloc(&s->slot_status, 64 * sizeof(int32_t), cudaHostAllocDefault));
  std::memset(s->slot_status, 0, 64 * sizeof(int32_t));
  for (uint32_t k = 0; k < 2 * slots; k++) {
    cudaStream_t st;
    QCB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    s->streams.push_back(st);
  }
  s->fill_gate = g_server_fill != 0;
  s->capacity = (uint32_t)std::max(device_sm_count(), 1);
  // keep this server's budget in the stream-ordered pool (the release
  // threshold grows by the budget while the server lives) and map it now:
  // growing the pool during serving maps fresh memory on the scheduler
  // thread (tens of ms for a multi-GB record) while it holds the lock
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t thr = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    thr = thr > UINT64_MAX - hbm_budget_bytes ? UINT64_MAX : thr + hbm_budget_bytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const uint64_t reserve = std::min<uint64_t>(hbm_budget_bytes, free_b > (1ull << 30) ? free_b - (1ull << 30) : 0);
    void* p = nullptr;
    if (reserve && cudaMallocAsync(&p, reserve, s->streams[0]) == cudaSuccess) {
      cudaFreeAsync(p, s->streams[0]);
      cudaStreamSynchronize(s->streams[0]);
    }
    cudaGetLastError();  // a reservation that did not fit is not an error
  }
  s->t0 = std::chrono::steady_clock::now();
  qcb_server* raw = s.get();
  s->th = std::thread(scheduler, raw);
  *out = s.release();
  return QCB_OK;
}

int qcb_server_submit(qcb_server* s, const qcb_op* ops, size_t n_ops, uint64_t shots, uint64_t seed,
                      uint64_t* ticket) {
  if (!s || !ticket || (n_ops && !ops)) return fail(QCB_EARG, "null argument");
  if (!shots) return fail(QCB_EARG, "serving: a request needs at least one shot");
  const double t_arrival = s->now();
  auto r = std::make_unique<Request>();
  r->ops.assign(ops, ops + n_ops);
  r->shots = shots;
  r->seed = seed;
  // the program: from the resident cache, else compiled here (in the
  // caller's thread, outside the server lock)
  const uint64_t h = ops_hash(r->ops);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (CachedProgram* c = find_program(s, h, r->ops)) {
      r->cached = c;
      c->refs++;  // held from here: eviction skips it
    }
  }
  if (!r->cached) {
    qcb_program* p = nullptr;
    if (int st = qcb_program_compile(r->ops.data(), r->ops.size(), &p)) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<qcb_op> key(r->ops);
    r->cached = insert_program(s, h, std::move(key), p);
    r->cached->refs++;
  }
  r->prog = r->cached->prog;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->cached->last_use = ++s->use_clock;
    r->id = s->next_id++;
    r->t_submit = t_arrival;
    *ticket = r->id;
    s->queue.push_back(r->id);
    s->reqs.emplace(r->id, std::move(r));
  }
  s->cv.notify_all();
  return QCB_OK;
}

// Compile a circuit into the resident program cache without running it.
int qcb_server_preload(qcb_server* s, const qcb_op* ops, size_t n_ops) {
  if (!s || (n_ops && !ops)) return fail(QCB_EARG, "null argument");
  std::vector<qcb_op> v(ops, ops + n_ops);
  const uint64_t h = ops_hash(v);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (CachedProgram* c = find_program(s, h, v)) {
      c->last_use = ++s->use_clock;
      return QCB_OK;
    }
  }
  qcb_program* p = nullptr;
  if (int st = qcb_program_compile(v.data(), v.size(), &p)) return st;
  std::lock_guard<std::mutex> lk(s->mu);
  insert_program(s, h, std::move(v), p)->last_use = ++s->use_clock;
  return QCB_OK;
}

// state: 0 queued, 1 running, 2 done, 3 failed; times (seconds since the
// server started): submit, admit, done.
int qcb_server_query(qcb_server* s, uint64_t ticket, int32_t* state, double* times3) {
  if (!s) return fail(QCB_EARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(QCB_EARG, "serving: unknown or released ticket");
  const Request& r = *it->second;
  if (state) *state = r.state;
  if (times3) { times3[0] = r.t_submit; times3[1] = r.t_admit; times3[2] = r.t_done; }
  return r.state == RQ_FAILED ? fail(r.status, r.msg) : QCB_OK;
}

// The next request that finished (or failed) and has not been reported yet,
// in completion order; blocks up to timeout_s.  state and times3 as for
// qcb_server_query.  QCB_ETIMEOUT when none finished in time.
int qcb_server_next_done(qcb_server* s, double timeout_s, uint64_t* ticket, int32_t* state, double* times3) {
  if (!s || !ticket) return fail(QCB_EARG, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  if (!s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return !s->completed.empty(); }))
    return fail(QCB_ETIMEOUT, "serving: no request finished within the timeout");
  const uint64_t id = s->completed.front();
  s->completed.pop_front();
  *ticket = id;
  auto it = s->reqs.find(id);
  if (it != s->reqs.end()) {
    const Request& r = *it->second;
    if (state) *state = r.state;
    if (times3) { times3[0] = r.t_submit; times3[1] = r.t_admit; times3[2] = r.t_done; }
  }
  return QCB_OK;
}

int qcb_server_wait(qcb_server* s, uint64_t ticket, double timeout_s) {
  if (!s) return fail(QCB_EARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto done = [&] {
    auto it = s->reqs.find(ticket);
    return it == s->reqs.end() || it->second->state >= RQ_DONE;
  };
  if (!s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
    return fail(QCB_ETIMEOUT, "serving: request not finished within the timeout");
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(QCB_EARG, "serving: unknown or released ticket");
  return it->second->state == RQ_FAILED ? fail(it->second->status, it->second->msg) : QCB_OK;
}

// The record of a finished request as shot-packed planes, nbits x
// ceil(shots/32) uint32 (host memory), where nbits is the program's.
int qcb_server_result(qcb_server* s, uint64_t ticket, uint32_t* planes, uint32_t* nbits_out) {
  if (!s) return fail(QCB_EARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(QCB_EARG, "serving: unknown or released ticket");
  Request& r = *it->second;
  if (r.state != RQ_DONE) return fail(QCB_EARG, "serving: request not finished");
  if (nbits_out) *nbits_out = r.prog->info.nbits;
  if (planes && r.prog->info.nbits)
    QCB_CUDA(cudaMemcpy2D(planes, r.ncols * 4, r.record, r.rec_pitch * 4, r.ncols * 4, r.prog->info.nbits,
                          cudaMemcpyDeviceToHost));
  return QCB_OK;
}

int qcb_server_release(qcb_server* s, uint64_t ticket) {
  if (!s) return fail(QCB_EARG, "null server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(QCB_EARG, "serving: unknown or released ticket");
    Request& r = *it->second;
    if (r.state < RQ_DONE) return fail(QCB_EARG, "serving: request still queued or running");
    if (r.record) {
      cudaFreeAsync(r.record, r.stream[0] ? r.stream[0] : s->streams[0]);  // the request's work is complete
      s->used -= r.bytes;
    }
    if (r.done) cudaEventDestroy(r.done);
    for (cudaEvent_t ev : r.chunk_ev)
      if (ev) cudaEventDestroy(ev);
    if (r.cached && r.cached->refs) r.cached->refs--;
    for (auto c = s->completed.begin(); c != s->completed.end(); ++c)
      if (*c == ticket) { s->completed.erase(c); break; }  // released without being reported
    s->reqs.erase(it);
  }
  s->cv.notify_all();  // memory freed: the scheduler may admit
  return QCB_OK;
}

int qcb_server_stats(qcb_server* s, uint64_t* used_bytes, uint64_t* program_bytes, uint32_t* n_programs) {
  if (!s) return fail(QCB_EARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (used_bytes) *used_bytes = s->used;
  if (program_bytes) *program_bytes = s->program_bytes;
  if (n_programs) *n_programs = (uint32_t)s->programs.size();
  return QCB_OK;
}

int qcb_server_destroy(qcb_server* s) {
  if (!s) return QCB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->th.joinable()) s->th.join();
  for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
  for (auto& kv : s->reqs) {
    if (kv.second->record) cudaFree(kv.second->record);
    for (qcb_frame* cf : kv.second->chunk) delete cf;
    if (kv.second->done) cudaEventDestroy(kv.second->done);
    for (cudaEvent_t ev : kv.second->chunk_ev)
      if (ev) cudaEventDestroy(ev);
  }
  if (s->slot_status) cudaFreeHost(s->slot_status);
  for (auto& kv : s->programs) qcb_program_destroy(kv.second->prog);
  for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t thr = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    thr = thr > s->budget ? thr - s->budget : 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  delete s;
  return QCB_OK;
}

}  // extern "C"
