// expect.cu -- expect(p, s) (src/project_trace_reset.jl:743-751) for many
// Paulis on one state, in one launch, without modifying the state.
//
// The reference computes project!(copy(s), p) and maps its result: nothing
// -> 0, 0x0 -> 1, 0x1 -> im, 0x2 -> -1, 0x3 -> -im.  On a copy, project! only
// has to say whether the Pauli anticommutes with a stabilizer (or a logical
// operator) -- result nothing -- and otherwise the phase of the Pauli it
// equals in the group:
//   * Destabilizer / MixedDestabilizer (src/project_trace_reset.jl:336-439):
//     the product of the stabilizer rows whose destabilizer anticommutes with
//     the Pauli, its phase starting at the Pauli's;
//   * Stabilizer / MixedStabilizer (:276-317): canonicalize! of the copy,
//     then generate! of the Pauli on it; canonicalize! is the same for every
//     Pauli, so it runs once on one copy.
// One warp per Pauli: lanes take 32 rows at a time for the commutation
// checks (the flags come out as ballots), and lanes take the words of a row
// for the products.  The stabilizer rows commute, so their product may be
// taken in any order with the same exact phase.
#include <algorithm>
#include <vector>

#include "qcb_internal.h"

namespace qcb {

int canonicalize_view(uint64_t* xzs, uint8_t* ph, uint32_t rows, uint32_t n, uint32_t W, int phases,
                      int32_t* d_out, cudaStream_t st);

__device__ __forceinline__ void mul_step_e(uint64_t x1, uint64_t z1, uint64_t& x2, uint64_t& z2, uint64_t& c1,
                                           uint64_t& c2) {
  const uint64_t nx = x1 ^ x2, nz = z1 ^ z2;
  const uint64_t x1z2 = x1 & z2;
  const uint64_t anti = (x2 & z1) ^ x1z2;
  c2 ^= (c1 ^ nx ^ nz ^ x1z2) & anti;
  c1 ^= anti;
  x2 = nx;
  z2 = nz;
}

// comm(P, row) of one row by one lane (src/QuantumClifford.jl:791-798).
__device__ __forceinline__ uint32_t row_comm(const uint64_t* P, const uint64_t* row, uint32_t len) {
  uint64_t acc = 0;
  for (uint32_t w = 0; w < len; w++) acc ^= (P[len + w] & row[w]) ^ (P[w] & row[len + w]);
  return (uint32_t)__popcll(acc) & 1u;
}

// Destabilizer kinds: rows [0, nn) destabilizers then logical X, [nn, 2nn)
// stabilizers then logical Z; r = rank.  out: -1 (nothing), else the phase.
__global__ void __launch_bounds__(256) expect_destab_kernel(const uint64_t* xzs, const uint8_t* ph, uint32_t nn,
                                                            uint32_t r, int mixed, uint32_t W,
                                                            const uint64_t* paulis, const uint8_t* pph,
                                                            uint32_t k, int32_t* out) {
  extern __shared__ __align__(16) uint64_t es[];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t len = W / 2;
  uint64_t* acc = es + (size_t)wib * W;  // this warp's product
  for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < k; j += nw) {
    const uint64_t* P = paulis + (size_t)j * W;
    // anticommutes with a stabilizer row, or (mixed) a logical row: nothing
    uint32_t anti = 0;
    for (uint32_t c = 0; c < 2 * nn && !anti; c += 32) {
      const uint32_t m = c + lane;
      uint32_t f = 0;
      const bool check = m < 2 * nn && ((m >= nn && m < nn + r) || (mixed && ((m >= r && m < nn) || m >= nn + r)));
      if (check) f = row_comm(P, xzs + (size_t)m * W, len);
      anti = __any_sync(0xFFFFFFFFu, f);
    }
    if (anti) {
      if (lane == 0) out[j] = -1;
      continue;
    }
    // the product of the stabilizer rows whose destabilizer anticommutes
    for (uint32_t w = lane; w < W; w += 32) acc[w] = 0;
    __syncwarp();
    uint64_t c1 = 0, c2 = 0;
    uint32_t extra = 0;
    for (uint32_t c = 0; c < r; c += 32) {
      const uint32_t i = c + lane;
      const uint32_t f = i < r ? row_comm(P, xzs + (size_t)i * W, len) : 0u;
      uint32_t mask = __ballot_sync(0xFFFFFFFFu, f);
      while (mask) {
        const uint32_t b = __ffs(mask) - 1;
        mask &= mask - 1;
        const uint64_t* srow = xzs + (size_t)(nn + c + b) * W;
        for (uint32_t w = lane; w < len; w += 32) {
          uint64_t x2 = acc[w], z2 = acc[len + w];
          mul_step_e(srow[w], srow[len + w], x2, z2, c1, c2);
          acc[w] = x2;
          acc[len + w] = z2;
        }
        extra += ph[nn + c + b];
      }
    }
    const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
    if (lane == 0) out[j] = (int32_t)((s + extra + pph[j]) & 3u);
    __syncwarp();
  }
}

// Stabilizer kinds on a canonical copy of the r rows: nothing if the Pauli
// anticommutes with a row, else generate! (src/project_trace_reset.jl:41-81):
// repeatedly the first set bit of the remaining Pauli (X half, then Z half),
// the first row at or after the last one used with that bit, and a product;
// a Pauli that is not reduced to the identity is not in the group (nothing).
__global__ void __launch_bounds__(256) expect_stab_kernel(const uint64_t* xzs, const uint8_t* ph, uint32_t r,
                                                          uint32_t W, const uint64_t* paulis,
                                                          const uint8_t* pph, uint32_t k, int32_t* out) {
  extern __shared__ __align__(16) uint64_t es[];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t len = W / 2;
  uint64_t* p = es + (size_t)wib * W;  // the remaining Pauli
  for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < k; j += nw) {
    const uint64_t* P = paulis + (size_t)j * W;
    uint32_t anti = 0;
    for (uint32_t c = 0; c < r && !anti; c += 32) {
      const uint32_t m = c + lane;
      anti = __any_sync(0xFFFFFFFFu, m < r ? row_comm(P, xzs + (size_t)m * W, len) : 0u);
    }
    if (anti) {
      if (lane == 0) out[j] = -1;
      continue;
    }
    for (uint32_t w = lane; w < W; w += 32) p[w] = P[w];
    __syncwarp();
    uint64_t c1 = 0, c2 = 0;
    uint32_t extra = pph[j], u = 0;
    bool good = true;
    for (uint32_t stage = 0; stage < 2 && good; stage++) {
      while (true) {
        uint32_t fb = 0xFFFFFFFFu;
        for (uint32_t w = lane; w < len; w += 32) {
          const uint64_t v = p[stage * len + w];
          if (v) fb = min(fb, w * 64 + (uint32_t)(__ffsll((long long)v) - 1));
        }
        fb = __reduce_min_sync(0xFFFFFFFFu, fb);
        if (fb == 0xFFFFFFFFu) break;
        const uint32_t ib = stage * len + (fb >> 6);
        const uint64_t bm = 1ull << (fb & 63);
        uint32_t cand = 0xFFFFFFFFu;
        for (uint32_t c = u; c < r && cand == 0xFFFFFFFFu; c += 32) {
          const uint32_t m = c + lane;
          const uint32_t hit = __ballot_sync(0xFFFFFFFFu, m < r && (xzs[(size_t)m * W + ib] & bm));
          if (hit) cand = c + __ffs(hit) - 1;
        }
        if (cand == 0xFFFFFFFFu) { good = false; break; }
        u = cand + 1;
        const uint64_t* l = xzs + (size_t)cand * W;
        for (uint32_t w = lane; w < len; w += 32) {
          uint64_t x2 = p[w], z2 = p[len + w];
          mul_step_e(l[w], l[len + w], x2, z2, c1, c2);
          p[w] = x2;
          p[len + w] = z2;
        }
        __syncwarp();
        extra += ph[cand];
      }
    }
    uint32_t nz = 0;
    for (uint32_t w = lane; w < W; w += 32) nz |= p[w] != 0;
    nz = __any_sync(0xFFFFFFFFu, nz);
    const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
    if (lane == 0) out[j] = (good && !nz) ? (int32_t)((s + extra) & 3u) : -1;
    __syncwarp();
  }
}

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_expect(const qcb_tableau* t, int kind, int32_t rank, const qcb_tableau* paulis, int32_t* out, void* stream) {
  if (!t || !paulis || !out) return fail(QCB_EARG, "null argument");
  if (paulis->nqubits != t->nqubits) return fail(QCB_EARG, "The number of qubits does not match");
  const uint32_t k = paulis->rows, W = t->W, n = t->nqubits;
  if (!k) return QCB_OK;
  cudaStream_t st = S(stream);
  int32_t* d_out = nullptr;
  QCB_CUDA(cudaMallocAsync(&d_out, (size_t)k * 4, st));
  const uint32_t threads = 256, wpb = threads / 32;
  const size_t sm = (size_t)wpb * W * 8;
  const uint32_t blocks = (uint32_t)std::min<uint64_t>((k + wpb - 1) / wpb, 16ull * device_sm_count());
  int status = QCB_OK;
  uint64_t* tmp = nullptr;
  uint8_t* tph = nullptr;
  if (kind == QCB_DESTABILIZER || kind == QCB_MIXED_DESTABILIZER) {
    if (t->rows % 2) { cudaFreeAsync(d_out, st); return fail(QCB_EDIM, "destabilizer tableaux have an even number of rows"); }
    const uint32_t nn = t->rows / 2;
    const bool mixed = kind == QCB_MIXED_DESTABILIZER;
    if (mixed && (rank < 0 || (uint32_t)rank > nn)) { cudaFreeAsync(d_out, st); return fail(QCB_EBOUNDS, "rank out of range"); }
    const uint32_t r = mixed ? (uint32_t)rank : nn;
    if (sm > 48 * 1024) QCB_CUDA(cudaFuncSetAttribute(expect_destab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    expect_destab_kernel<<<blocks, threads, sm, st>>>(t->xzs, t->phases, nn, r, mixed ? 1 : 0, W, paulis->xzs,
                                                       paulis->phases, k, d_out);
    QCB_LAUNCHED();
    if (!mixed && nn != n) status = QCB_EBADSTRUCT;  // decided per Pauli below
  } else if (kind == QCB_STABILIZER || kind == QCB_MIXED_STABILIZER) {
    const bool mixed = kind == QCB_MIXED_STABILIZER;
    if (mixed && (rank < 0 || (uint32_t)rank > t->rows)) { cudaFreeAsync(d_out, st); return fail(QCB_EBOUNDS, "rank out of range"); }
    const uint32_t r = mixed ? (uint32_t)rank : t->rows;
    // canonicalize! of one copy of the stabilizer rows
    QCB_CUDA(cudaMallocAsync(&tmp, std::max<size_t>((size_t)r * W * 8, 8), st));
    QCB_CUDA(cudaMallocAsync(&tph, std::max<uint32_t>(r, 1), st));
    if (r) {
      QCB_CUDA(cudaMemcpyAsync(tmp, t->xzs, (size_t)r * W * 8, cudaMemcpyDeviceToDevice, st));
      QCB_CUDA(cudaMemcpyAsync(tph, t->phases, r, cudaMemcpyDeviceToDevice, st));
      status = canonicalize_view(tmp, tph, r, n, W, 1, (int32_t*)t->scratch + 48, st);
    }
    if (status == QCB_OK) {
      if (sm > 48 * 1024) QCB_CUDA(cudaFuncSetAttribute(expect_stab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      expect_stab_kernel<<<blocks, threads, sm, st>>>(tmp, tph, r, W, paulis->xzs, paulis->phases, k, d_out);
      QCB_LAUNCHED();
    }
  } else {
    cudaFreeAsync(d_out, st);
    return fail(QCB_EARG, "expect: bad state kind");
  }
  std::vector<int32_t> h(k, -1);
  if (status == QCB_OK || status == QCB_EBADSTRUCT) {
    if (cudaMemcpyAsync(h.data(), d_out, (size_t)k * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) status = fail(QCB_ECUDA, "expect: copy");
  }
  cudaFreeAsync(d_out, st);
  if (tmp) cudaFreeAsync(tmp, st);
  if (tph) cudaFreeAsync(tph, st);
  QCB_CUDA(cudaStreamSynchronize(st));
  if (status == QCB_EBADSTRUCT) {
    // an incomplete Destabilizer cannot decide a commuting Pauli
    for (uint32_t j = 0; j < k; j++)
      if (h[j] >= 0)
        return fail(QCB_EBADSTRUCT,
                    "`Destabilizer` can not efficiently (faster than n^3) detect whether you are projecting on a "
                    "stabilized or a logical operator. Switch to one of the `Mixed*` data structures.");
    status = QCB_OK;
  }
  if (status != QCB_OK) return status;
  std::copy(h.begin(), h.end(), out);
  return QCB_OK;
}

}  // extern "C"
