// server.cu -- the serving loop: sampling requests submitted at any time, kept
// resident on the device and run with continuous batching.
//
// A request is a circuit (op list), a shot count and a seed.  Its program is
// compiled once per distinct op list and stays resident (a cache keyed by
// the op bytes).  Admission is first come, first served against an HBM
// budget and a number of slots: the head of the queue is admitted as soon as
// a slot is free and its memory (the full record, plus one chunk's frame
// planes) fits the budget.  Device memory comes from the stream-ordered
// allocator (cudaMallocAsync / cudaFreeAsync on the slot's stream), so the
// scheduler thread never waits for the device.  An admitted request runs on its
// slot's stream as a sequence of shot chunks (fresh Philox runs with the
// chunk's global shot offset, each writing its columns of the request's
// record), so requests admitted while others run share the GPU chunk by
// chunk, and every record equals that of one plain run of the request.  A
// scheduler thread admits, launches and retires (CUDA events); the caller
// polls, waits, copies results out and releases them.
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

struct Request {
  uint64_t id = 0;
  std::vector<qcb_op> ops;
  uint64_t shots = 0, seed = 0;
  qcb_program* prog = nullptr;  // cached, owned by the server
  uint64_t nbits = 0, ncols = 0, rec_pitch = 0;
  uint64_t bytes = 0;           // record + chunk planes charged to the budget
  uint32_t* record = nullptr;
  qcb_frame* chunk = nullptr;   // the chunk frame (its planes live while the chunks run)
  int slot = -1;
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
  std::vector<cudaStream_t> streams;
  std::vector<int64_t> slot_req;  // request id per slot, -1 when free
  std::map<uint64_t, std::unique_ptr<qcb::Request>> reqs;
  std::deque<uint64_t> queue;
  std::deque<uint64_t> completed;  // finished or failed, not yet reported by next_done
  std::unordered_map<uint64_t, qcb_program*> programs;
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

static uint64_t ops_hash(const std::vector<qcb_op>& ops) {
  uint64_t h = 1469598103934665603ull;
  const uint8_t* p = (const uint8_t*)ops.data();
  for (size_t i = 0; i < ops.size() * sizeof(qcb_op); i++) { h ^= p[i]; h *= 1099511628211ull; }
  return h ^ (ops.size() * 0x9E3779B97F4A7C15ull);
}

static uint64_t chunk_plane_bytes(uint32_t nq1, uint64_t chunk_cols) {
  const uint64_t pitch = std::max<uint64_t>(32, (chunk_cols + 31) / 32 * 32);
  return (uint64_t)2 * (nq1 + 1) * pitch * 4 + (uint64_t)pitch * 4 + 16;
}

// Admit the head of the queue while a slot and the budget allow (called
// with the lock held).  Returns after launching every chunk of each admitted
// request on its slot's stream.
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
      r.bytes = r.nbits * r.rec_pitch * 4 + chunk_plane_bytes(std::max<uint32_t>(r.prog->nq, 1), s->chunk_cols);
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
    if (s->used + r.bytes > s->budget) return;  // first come, first served: wait for memory
    const uint32_t nq1 = std::max<uint32_t>(r.prog->nq, 1);
    cudaStream_t st = s->streams[slot];
    // the chunk frame: planes for one chunk, allocated and freed in stream
    // order (no device-wide synchronisation on the scheduler thread)
    qcb_frame* cf = new qcb_frame();
    cf->frames = s->chunk_cols * 32;
    cf->qubits = nq1 - 1;
    cf->nq1 = nq1;
    cf->nbits = 0;
    cf->ncols = s->chunk_cols;
    cf->pitch = std::max<uint64_t>(32, (s->chunk_cols + 31) / 32 * 32);
    cf->planes = nullptr;
    cf->record = nullptr;
    cf->err = nullptr;
    r.chunk = cf;
    cudaError_t e = cudaMallocAsync(&cf->planes, (size_t)2 * (nq1 + 1) * cf->pitch * 4, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&cf->err, 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cf->err, 0, 16, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&r.record, r.nbits * r.rec_pitch * 4, st);
    if (e == cudaSuccess && !r.done) e = cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming);
    int status = e == cudaSuccess ? QCB_OK : cuda_fail(e, "serving: admission");
    for (uint64_t c0 = 0; status == QCB_OK && c0 < r.ncols; c0 += s->chunk_cols) {
      const uint64_t nc = std::min<uint64_t>(s->chunk_cols, r.ncols - c0);
      status = run_chunk(r.chunk, nc, r.prog, r.seed, c0 * 32, r.record + c0, r.rec_pitch, st);
    }
    if (status == QCB_OK &&
        cudaMemcpyAsync(&s->slot_status[slot], cf->err, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      status = fail(QCB_ECUDA, "serving: status copy");
    if (cf->planes) cudaFreeAsync(cf->planes, st);
    if (cf->err) cudaFreeAsync(cf->err, st);
    cf->planes = nullptr;
    cf->err = nullptr;
    if (status == QCB_OK && cudaEventRecord(r.done, st) != cudaSuccess) status = fail(QCB_ECUDA, "serving: event");
    s->queue.pop_front();
    r.t_admit = s->now();
    if (status != QCB_OK) {
      r.msg = last_msg();
      if (r.record) cudaFreeAsync(r.record, st);
      r.record = nullptr;
      delete r.chunk;
      r.chunk = nullptr;
      r.state = RQ_FAILED; r.status = status; r.t_done = s->now();
      s->completed.push_back(r.id);
      s->done_cv.notify_all();
      continue;
    }
    r.slot = slot;
    r.state = RQ_RUNNING;
    s->slot_req[slot] = (int64_t)r.id;
    s->used += r.bytes;
  }
}

// Retire the running requests whose last chunk has finished (lock held):
// their chunk planes were freed in stream order, their records stay until
// released.
static void retire(qcb_server* s) {
  for (uint32_t k = 0; k < s->nslots; k++) {
    if (s->slot_req[k] < 0) continue;
    Request& r = *s->reqs[(uint64_t)s->slot_req[k]];
    const cudaError_t q = cudaEventQuery(r.done);
    if (q == cudaErrorNotReady) continue;
    r.t_done = s->now();
    r.state = q == cudaSuccess ? RQ_DONE : RQ_FAILED;
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
    delete r.chunk;
    r.chunk = nullptr;
    // the chunk planes leave the request's charge; the record stays charged
    s->used -= chunk_plane_bytes(std::max<uint32_t>(r.prog->nq, 1), s->chunk_cols);
    r.bytes -= chunk_plane_bytes(std::max<uint32_t>(r.prog->nq, 1), s->chunk_cols);
    s->slot_req[k] = -1;
    s->completed.push_back(r.id);
    s->done_cv.notify_all();
  }
}

static void scheduler(qcb_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
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
  for (uint32_t k = 0; k < slots; k++) {
    cudaStream_t st;
    QCB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    s->streams.push_back(st);
  }
  // keep freed record memory in the stream-ordered pool up to the budget
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t thr = hbm_budget_bytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
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
    auto it = s->programs.find(h);
    if (it != s->programs.end()) r->prog = it->second;
  }
  if (!r->prog) {
    qcb_program* p = nullptr;
    if (int st = qcb_program_compile(r->ops.data(), r->ops.size(), &p)) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    auto ins = s->programs.emplace(h, p);
    if (!ins.second) qcb_program_destroy(p);
    r->prog = ins.first->second;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
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
    if (s->programs.count(h)) return QCB_OK;
  }
  qcb_program* p = nullptr;
  if (int st = qcb_program_compile(v.data(), v.size(), &p)) return st;
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->programs.emplace(h, p).second) qcb_program_destroy(p);
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
      cudaFreeAsync(r.record, s->streams[r.slot >= 0 ? r.slot : 0]);  // the request's work is complete
      s->used -= r.bytes;
    }
    if (r.done) cudaEventDestroy(r.done);
    for (auto c = s->completed.begin(); c != s->completed.end(); ++c)
      if (*c == ticket) { s->completed.erase(c); break; }  // released without being reported
    s->reqs.erase(it);
  }
  s->cv.notify_all();  // memory freed: the scheduler may admit
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
    delete kv.second->chunk;
    if (kv.second->done) cudaEventDestroy(kv.second->done);
  }
  if (s->slot_status) cudaFreeHost(s->slot_status);
  for (auto& kv : s->programs) qcb_program_destroy(kv.second);
  for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
  delete s;
  return QCB_OK;
}

}  // extern "C"
