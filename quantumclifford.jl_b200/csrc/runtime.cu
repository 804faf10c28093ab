// runtime.cu -- library state, errors, tableau storage, diagnostics.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "qcb_internal.h"

namespace qcb {

std::atomic<uint64_t> g_launches{0};
static thread_local int t_status = QCB_OK;
static thread_local std::string t_msg;

void set_error(int status, const std::string& msg) {
  t_status = status;
  t_msg = msg;
}

int fail(int status, const std::string& msg) {
  set_error(status, msg);
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  int st = (e == cudaErrorMemoryAllocation) ? QCB_EOOM : QCB_ECUDA;
  return fail(st, m);
}

int device_sm_count() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 1;
}

int device_max_smem_optin() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v > 0 ? v : 48 * 1024;
}

__global__ void philox_probe_kernel(uint4 ctr, uint2 key, uint32_t* out) {
  uint32_t o[4];
  philox4x32_10(ctr.x, ctr.y, ctr.z, ctr.w, key.x, key.y, o);
  for (int i = 0; i < 4; i++) out[i] = o[i];
}

void set_walker_tile(uint32_t t);
void set_walker_threads(uint32_t t);
void set_stage_withhold(uint32_t k);
void set_presample(uint32_t v);
void set_server_hash_bits(uint32_t b);
void set_canon_cluster(uint32_t cs);
void set_canon_threads(uint32_t n);
void set_project_cluster(uint32_t cs);
void set_project_grid(uint32_t v);
void set_project_withhold(uint32_t v);
void set_canon_blocked(uint32_t v);
void set_canon_grid(uint32_t v);
void set_server_fill(uint32_t v);
void set_canon_rpt(uint32_t v);
void set_canon_pdl(uint32_t v);
void set_gates_pdl(uint32_t v);
void set_canon_lookahead(uint32_t v);
void set_walker_pdl(uint32_t v);
void set_walker_narrow(uint32_t v);
void set_canon_apply_rows(uint32_t v);

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_init(int device) {
  int n = 0;
  QCB_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(QCB_EBOUNDS, "qcb_init: no such device");
  QCB_CUDA(cudaSetDevice(device));
  QCB_CUDA(cudaFree(0));
  // keep up to 1 GB of freed stream-ordered memory in the device's default
  // pool: the per-call scratch of the tableau kernels (cudaMallocAsync /
  // cudaFreeAsync) is then taken from the pool instead of being mapped
  // through the driver on every call (with the default threshold of 0 the
  // pool returns it at each synchronisation)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if (thr < (1ull << 30)) {
      thr = 1ull << 30;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  return QCB_OK;
}

const char* qcb_version(void) { return "qcb200 0.1.0 (sm_100a)"; }

int qcb_last_error(char* buf, size_t len) {
  if (buf && len) {
    std::snprintf(buf, len, "%s", t_msg.c_str());
  }
  return t_status;
}

const char* qcb_status_string(int s) {
  switch (s) {
    case QCB_OK: return "QCB_OK";
    case QCB_EDIM: return "QCB_EDIM";
    case QCB_EBOUNDS: return "QCB_EBOUNDS";
    case QCB_EZEROQUBIT: return "QCB_EZEROQUBIT";
    case QCB_EARG: return "QCB_EARG";
    case QCB_EOOM: return "QCB_EOOM";
    case QCB_EBUDGET: return "QCB_EBUDGET";
    case QCB_ETIMEOUT: return "QCB_ETIMEOUT";
    case QCB_ECUDA: return "QCB_ECUDA";
    case QCB_EBADSTRUCT: return "QCB_EBADSTRUCT";
    case QCB_EUNSUPPORTED: return "QCB_EUNSUPPORTED";
    case QCB_ENOTREADY: return "QCB_ENOTREADY";
    default: return "QCB_UNKNOWN";
  }
}

int qcb_device_synchronize(void) {
  QCB_CUDA(cudaDeviceSynchronize());
  return QCB_OK;
}

uint64_t qcb_launch_count(void) { return g_launches.load(); }

int qcb_tune_set(const char* key, int64_t value) {
  if (!key) return fail(QCB_EARG, "qcb_tune_set: null key");
  const std::string k(key);
  if (value < 0 || value > 1024) return fail(QCB_EARG, "qcb_tune_set: value out of range");
  if (k == "walker_tile") {
    if (value && (value < 8 || value > 256 || value % 2)) return fail(QCB_EARG, "walker_tile must be 0 (automatic) or even, 8..256");
    set_walker_tile((uint32_t)value);
  } else if (k == "stage_withhold") {
    // test knob: the plain walker never stages window `value` (1-based count
    // of each CTA's window sequence), so its bounded wait expires and the run
    // reports QCB_ETIMEOUT; 0 turns it off
    set_stage_withhold((uint32_t)value);
  } else if (k == "presample") {
    // 0: the noise of Philox runs is drawn by the pre-sampler where its
    // scratch fits; 1: always in the walk; 2 (test): pre-sampled, but every
    // bucket reports an overflow, so the walk draws them (the fallback path)
    if (value > 2) return fail(QCB_EARG, "presample must be 0, 1 or 2");
    set_presample((uint32_t)value);
  } else if (k == "server_hash_bits") {
    // test knob: the serving program cache keeps only `value` low bits of
    // its hash (0: all), so that distinct circuits collide
    if (value > 64) return fail(QCB_EARG, "server_hash_bits must be 0..64");
    set_server_hash_bits((uint32_t)value);
  } else if (k == "server_fill") {
    // serving admission: 1 (default) onto idle SMs only, 0 whenever a slot is
    // free; read when a server is created
    if (value > 1) return fail(QCB_EARG, "server_fill must be 0 or 1");
    set_server_fill((uint32_t)value);
  } else if (k == "walker_threads") {
    if (value && (value < 64 || value > 640 || value % 32)) return fail(QCB_EARG, "walker_threads must be 0 (640) or 64..640, a multiple of 32");
    set_walker_threads((uint32_t)value);
  } else if (k == "canon_threads") {
    if (value && (value < 64 || value > 1024 || value % 32)) return fail(QCB_EARG, "canon_threads must be 0 or 64..1024, a multiple of 32");
    set_canon_threads((uint32_t)value);
  } else if (k == "canon_cluster") {
    if (value && (value > 16 || (value & (value - 1)))) return fail(QCB_EARG, "canon_cluster must be 1, 2, 4, 8 or 16");
    set_canon_cluster((uint32_t)value);
  } else if (k == "canon_blocked") {
    if (value > 2) return fail(QCB_EARG, "canon_blocked must be 0 (automatic), 1 (always) or 2 (never)");
    set_canon_blocked((uint32_t)value);
  } else if (k == "canon_grid") {
    // canonicalize! by panels over the whole GPU: 0 from 640 rows, 1 always, 2 never
    if (value > 2) return fail(QCB_EARG, "canon_grid must be 0 (automatic), 1 (always) or 2 (never)");
    set_canon_grid((uint32_t)value);
  } else if (k == "canon_rpt") {
    if (value && value != 1 && value != 2 && value != 4 && value != 8 && value != 16)
      return fail(QCB_EARG, "canon_rpt must be 0, 1, 2, 4, 8 or 16");
    set_canon_rpt((uint32_t)value);
  } else if (k == "walker_narrow") {
    // tall programs whose 16-column tile does not fit shared memory: 8..14-
    // column tiles (1, default) or the walker on the HBM planes (0)
    if (value > 1) return fail(QCB_EARG, "walker_narrow must be 0 or 1");
    set_walker_narrow((uint32_t)value);
  } else if (k == "walker_pdl") {
    // the frame walker as a programmatic dependent of the noise pre-sampler (1, default) or plain (0)
    if (value > 1) return fail(QCB_EARG, "walker_pdl must be 0 or 1");
    set_walker_pdl((uint32_t)value);
  } else if (k == "canon_pdl") {
    // canonicalize! panel launches as programmatic dependents (1, default) or plain (0)
    if (value > 1) return fail(QCB_EARG, "canon_pdl must be 0 or 1");
    set_canon_pdl((uint32_t)value);
  } else if (k == "canon_lookahead") {
    // canonicalize! by panels over the whole GPU: the next panel's pivot
    // steps beside this panel's apply (1, default) or the two in turn (0)
    if (value > 1) return fail(QCB_EARG, "canon_lookahead must be 0 or 1");
    set_canon_lookahead((uint32_t)value);
  } else if (k == "gates_pdl") {
    // symbolic apply! launches (qcb_apply_gates) as programmatic dependents (1, default) or plain (0)
    if (value > 1) return fail(QCB_EARG, "gates_pdl must be 0 or 1");
    set_gates_pdl((uint32_t)value);
  } else if (k == "canon_apply_rows") {
    if (value && (value < 8 || value > 32)) return fail(QCB_EARG, "canon_apply_rows must be 0 or 8..32");
    set_canon_apply_rows((uint32_t)value);
  } else if (k == "project_grid") {
    // project! of generic Paulis on Stabilizer / MixedStabilizer tableaux on
    // the whole GPU: 0 when the tableau does not fit one cluster's shared
    // memory, 1 always, 2 never
    if (value > 2) return fail(QCB_EARG, "project_grid must be 0, 1 or 2");
    set_project_grid((uint32_t)value);
  } else if (k == "project_withhold") {
    // test knob: one CTA of the whole-GPU project! kernel leaves before the
    // first grid barrier, so the others' bounded waits run out and the call
    // returns QCB_ETIMEOUT (nothing faults)
    if (value > 1) return fail(QCB_EARG, "project_withhold must be 0 or 1");
    set_project_withhold((uint32_t)value);
  } else if (k == "project_cluster") {
    if (value && (value > 16 || (value & (value - 1)))) return fail(QCB_EARG, "project_cluster must be 1, 2, 4, 8 or 16");
    set_project_cluster((uint32_t)value);
  } else {
    return fail(QCB_EARG, "qcb_tune_set: unknown key " + k);
  }
  return QCB_OK;
}

int qcb_debug_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t* d = nullptr;
  QCB_CUDA(cudaMalloc(&d, 16));
  philox_probe_kernel<<<1, 1>>>(make_uint4(ctr[0], ctr[1], ctr[2], ctr[3]),
                                make_uint2(key[0], key[1]), d);
  g_launches.fetch_add(1);
  cudaError_t e = cudaMemcpy(out, d, 16, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "qcb_debug_philox");
  return QCB_OK;
}

// ------------------------------------------------------------ tableaux
int qcb_tableau_create(uint32_t rows, uint32_t nqubits, qcb_tableau** out) {
  if (!out) return fail(QCB_EARG, "qcb_tableau_create: null out");
  *out = nullptr;
  qcb_tableau* t = new qcb_tableau();
  t->rows = rows;
  t->nqubits = nqubits;
  t->W = 2 * ((nqubits + 63) / 64);
  size_t words = (size_t)rows * t->W;
  cudaError_t e = cudaMalloc(&t->xzs, (words ? words : 1) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&t->phases, rows ? rows : 1);
  if (e == cudaSuccess) e = cudaMalloc(&t->scratch, 4096);
  if (e == cudaSuccess) e = cudaMemset(t->xzs, 0, (words ? words : 1) * 8);
  if (e == cudaSuccess) e = cudaMemset(t->phases, 0, rows ? rows : 1);
  if (e == cudaSuccess) e = cudaMemset(t->scratch, 0, 4096);
  if (e != cudaSuccess) {
    cudaFree(t->xzs); cudaFree(t->phases); cudaFree(t->scratch);
    delete t;
    return cuda_fail(e, "qcb_tableau_create");
  }
  *out = t;
  return QCB_OK;
}

int qcb_tableau_destroy(qcb_tableau* t) {
  if (!t) return QCB_OK;
  cudaFree(t->xzs);
  cudaFree(t->phases);
  cudaFree(t->scratch);
  delete t;
  return QCB_OK;
}

int qcb_tableau_shape(const qcb_tableau* t, uint32_t* rows, uint32_t* nqubits) {
  if (!t) return fail(QCB_EARG, "null tableau");
  if (rows) *rows = t->rows;
  if (nqubits) *nqubits = t->nqubits;
  return QCB_OK;
}

int qcb_tableau_upload(qcb_tableau* t, const uint8_t* phases, const uint64_t* xzs, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  size_t words = (size_t)t->rows * t->W;
  if (xzs && words) QCB_CUDA(cudaMemcpyAsync(t->xzs, xzs, words * 8, cudaMemcpyHostToDevice, S(stream)));
  if (phases && t->rows) QCB_CUDA(cudaMemcpyAsync(t->phases, phases, t->rows, cudaMemcpyHostToDevice, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_tableau_download(const qcb_tableau* t, uint8_t* phases, uint64_t* xzs, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  size_t words = (size_t)t->rows * t->W;
  if (xzs && words) QCB_CUDA(cudaMemcpyAsync(xzs, t->xzs, words * 8, cudaMemcpyDeviceToHost, S(stream)));
  if (phases && t->rows) QCB_CUDA(cudaMemcpyAsync(phases, t->phases, t->rows, cudaMemcpyDeviceToHost, S(stream)));
  QCB_CUDA(cudaStreamSynchronize(S(stream)));
  return QCB_OK;
}

int qcb_tableau_copy(qcb_tableau* dst, const qcb_tableau* src, void* stream) {
  if (!dst || !src) return fail(QCB_EARG, "null tableau");
  if (dst->rows != src->rows || dst->nqubits != src->nqubits)
    return fail(QCB_EDIM, "qcb_tableau_copy: shapes differ");
  size_t words = (size_t)src->rows * src->W;
  if (words) QCB_CUDA(cudaMemcpyAsync(dst->xzs, src->xzs, words * 8, cudaMemcpyDeviceToDevice, S(stream)));
  if (src->rows) QCB_CUDA(cudaMemcpyAsync(dst->phases, src->phases, src->rows, cudaMemcpyDeviceToDevice, S(stream)));
  return QCB_OK;
}

}  // extern "C"
