// canon.cu -- canonicalize! and generate! on device tableaux.
//
// canonicalize! (src/canonicalization.jl:95-133) is Garcia's two-stage
// elimination: for every column j (X bits, then Z bits) find the first row at
// or below the current pivot position i with the bit set, swap it to i, and
// left-multiply every other row that has the bit by the pivot row.  The
// pivot steps are serial, so the kernel is one thread-block cluster that stays
// resident for the whole elimination:
//   - the rows are split over the cluster's CTAs and held in shared memory
//     (row stride W+1 words, so a thread-per-row column probe and a
//     warp-per-row update are both bank-conflict free); tableaux too tall for
//     the cluster's shared memory stay in global memory (L2) instead;
//   - rows never move: a row swap only exchanges logical positions (pos[] per
//     CTA, inv[] replicated in every CTA), and rows are written to their final
//     positions at the end;
//   - per column each CTA reduces its local candidate (smallest position >= i
//     with the bit) with __reduce_min_sync, publishes it in shared memory, and
//     after one cluster barrier every CTA reads all candidates through
//     distributed shared memory; the pivot row is fetched the same way.
// The row products keep the reference's phase arithmetic exactly
// (mul_left!(state, m, i): phase_m <- (s + phase_m + phase_i) mod 4).
#include <cooperative_groups.h>

#include <algorithm>

#include "qcb_internal.h"

namespace cg = cooperative_groups;

namespace qcb {

__device__ __forceinline__ void mul_step_c(uint64_t x1, uint64_t z1, uint64_t& x2, uint64_t& z2,
                                           uint64_t& c1, uint64_t& c2) {
  const uint64_t nx = x1 ^ x2, nz = z1 ^ z2;
  const uint64_t x1z2 = x1 & z2;
  const uint64_t anti = (x2 & z1) ^ x1z2;
  c2 ^= (c1 ^ nx ^ nz ^ x1z2) & anti;
  c1 ^= anti;
  x2 = nx;
  z2 = nz;
}

struct CanonArgs {
  uint64_t* xzs;   // first row of the view
  uint8_t* ph;
  uint32_t rows, n, W;
  uint32_t RB;     // rows per CTA
  int phases;
  int smem_rows;   // 1: rows staged in shared memory
  uint64_t* gtmp;  // global mode: permuted output
  uint8_t* gtmp_ph;
  int32_t* out;    // rx, rz
};

constexpr uint32_t CANON_THREADS = 1024;

__global__ void __launch_bounds__(CANON_THREADS) canon_kernel(const CanonArgs a) {
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t me = cl.block_rank();
  const uint32_t CS = cl.num_blocks();
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t W = a.W, len = W / 2, WS = W + 1;
  const uint32_t r0 = me * a.RB;
  const uint32_t nloc = r0 < a.rows ? min(a.RB, a.rows - r0) : 0u;

  extern __shared__ __align__(16) uint64_t smem[];
  uint64_t* piv = smem;                                   // W words
  uint64_t* rowsbuf = piv + W + 1;                        // RB * WS words (smem mode)
  uint8_t* bytes = (uint8_t*)(rowsbuf + (a.smem_rows ? (size_t)a.RB * WS : 0));
  uint32_t* slot = (uint32_t*)bytes;                      // 2 candidate slots
  uint32_t* red = slot + 2;                               // 32 warp minima
  uint32_t* ctl = red + 32;                               // [0]=k [1]=pstar [2]=piv phase
  uint32_t* inv = ctl + 4;                                // rows (replicated)
  uint32_t* pos = inv + a.rows;                           // RB
  uint8_t* lph = (uint8_t*)(pos + a.RB);                  // RB

  auto ROW = [&](uint32_t r) -> uint64_t* {
    return a.smem_rows ? rowsbuf + (size_t)r * WS : a.xzs + (size_t)(r0 + r) * W;
  };

  for (uint32_t r = tid; r < nloc; r += blockDim.x) {
    pos[r] = r0 + r;
    lph[r] = a.ph[r0 + r];
  }
  if (a.smem_rows) {
    for (uint32_t r = warp; r < nloc; r += nwarps)
      for (uint32_t w = lane; w < W; w += 32) rowsbuf[(size_t)r * WS + w] = a.xzs[(size_t)(r0 + r) * W + w];
  }
  for (uint32_t p = tid; p < a.rows; p += blockDim.x) inv[p] = p;
  cl.sync();

  uint32_t i = 0, step = 0, rx = 0;
  for (uint32_t stage = 0; stage < 2; stage++) {
    for (uint32_t j = 0; j < a.n; j++, step++) {
      const uint32_t wj = stage * len + (j >> 6);
      const uint64_t bm = 1ull << (j & 63);
      // local candidate: smallest position >= i with the bit set
      uint32_t best = 0xFFFFFFFFu;
      for (uint32_t r = tid; r < nloc; r += blockDim.x) {
        const uint32_t p = pos[r];
        if (p >= i && (ROW(r)[wj] & bm)) best = min(best, p);
      }
      best = __reduce_min_sync(0xFFFFFFFFu, best);
      if (lane == 0) red[warp] = best;
      __syncthreads();
      if (warp == 0) {
        uint32_t b = lane < nwarps ? red[lane] : 0xFFFFFFFFu;
        b = __reduce_min_sync(0xFFFFFFFFu, b);
        if (lane == 0) slot[step & 1] = b;
      }
      cl.sync();
      if (warp == 0) {
        // the cluster's candidates, one CTA per lane
        uint32_t k = lane < CS ? *cl.map_shared_rank(&slot[step & 1], lane) : 0xFFFFFFFFu;
        k = __reduce_min_sync(0xFFFFFFFFu, k);
        if (lane == 0) ctl[0] = k;
        if (lane == 0 && k != 0xFFFFFFFFu) {
          // rowswap!(state, k, i) on logical positions
          const uint32_t pstar = inv[k], aphys = inv[i];
          inv[i] = pstar;
          inv[k] = aphys;
          if (pstar >= r0 && pstar < r0 + nloc) pos[pstar - r0] = i;
          if (aphys >= r0 && aphys < r0 + nloc) pos[aphys - r0] = k;
          ctl[1] = pstar;
        }
      }
      __syncthreads();
      const uint32_t k = ctl[0];
      if (k == 0xFFFFFFFFu) continue;
      const uint32_t pstar = ctl[1];
      const uint32_t owner = pstar / a.RB, lr = pstar - owner * a.RB;
      {
        const uint64_t* src;
        const uint8_t* srcph;
        if (a.smem_rows) {
          uint64_t* base = rowsbuf + (size_t)lr * WS;
          uint8_t* pb = lph + lr;
          src = owner == me ? base : cl.map_shared_rank(base, owner);
          srcph = owner == me ? pb : cl.map_shared_rank(pb, owner);
        } else {
          src = a.xzs + (size_t)pstar * W;
          uint8_t* pb = lph + lr;
          srcph = owner == me ? pb : cl.map_shared_rank(pb, owner);
        }
        for (uint32_t w = tid; w < W; w += blockDim.x) piv[w] = src[w];
        if (tid == 0) ctl[2] = *srcph;
      }
      __syncthreads();
      const uint32_t pph = ctl[2];
      for (uint32_t r = warp; r < nloc; r += nwarps) {
        if (r0 + r == pstar) continue;
        uint64_t* row = ROW(r);
        if (!(row[wj] & bm)) continue;
        uint64_t c1 = 0, c2 = 0;
        for (uint32_t w = lane; w < len; w += 32) {
          uint64_t x2 = row[w], z2 = row[len + w];
          mul_step_c(piv[w], piv[len + w], x2, z2, c1, c2);
          row[w] = x2;
          row[len + w] = z2;
        }
        if (a.phases) {
          const uint32_t s =
              __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
          if (lane == 0) lph[r] = (uint8_t)((s + lph[r] + pph) & 3u);
        }
      }
      __syncthreads();
      i++;
    }
    if (stage == 0) rx = i;
  }
  // every CTA is done reading remote shared memory before anyone leaves
  cl.sync();
  if (a.smem_rows) {
    for (uint32_t r = warp; r < nloc; r += nwarps) {
      const uint32_t p = pos[r];
      for (uint32_t w = lane; w < W; w += 32) a.xzs[(size_t)p * W + w] = rowsbuf[(size_t)r * WS + w];
      if (lane == 0 && a.phases) a.ph[p] = lph[r];
    }
  } else {
    for (uint32_t r = warp; r < nloc; r += nwarps) {
      const uint32_t p = pos[r];
      for (uint32_t w = lane; w < W; w += 32) a.gtmp[(size_t)p * W + w] = a.xzs[(size_t)(r0 + r) * W + w];
      if (lane == 0) a.gtmp_ph[p] = a.phases ? lph[r] : a.ph[p];
    }
  }
  if (me == 0 && tid == 0) {
    a.out[0] = (int32_t)rx;
    a.out[1] = (int32_t)i;
  }
}

// generate! (src/project_trace_reset.jl:41-81) on a canonical stabilizer,
// one CTA.  The Pauli lives in shared memory; each step finds the first set
// bit, the first usable row with that bit, and multiplies.
__global__ void __launch_bounds__(1024) generate_kernel(uint64_t* pauli, uint8_t* pph,
                                                        const uint64_t* xzs, const uint8_t* ph,
                                                        uint32_t rows, uint32_t W, int phases,
                                                        int32_t* ok, int32_t* used, uint32_t cap,
                                                        uint32_t* n_used) {
  extern __shared__ __align__(16) uint64_t gs[];
  uint64_t* p = gs;
  __shared__ uint32_t red[32];
  __shared__ uint32_t sh[4];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t len = W / 2;
  for (uint32_t w = tid; w < W; w += blockDim.x) p[w] = pauli[w];
  if (tid == 0) { sh[2] = pph[0]; sh[3] = 0; }
  __syncthreads();
  uint32_t u = 0, nu = 0, good = 1;
  for (uint32_t stage = 0; stage < 2 && good; stage++) {
    while (true) {
      // first set bit of this half
      uint32_t fb = 0xFFFFFFFFu;
      for (uint32_t w = tid; w < len; w += blockDim.x) {
        const uint64_t v = p[stage * len + w];
        if (v) fb = min(fb, w * 64 + (uint32_t)(__ffsll((long long)v) - 1));
      }
      fb = __reduce_min_sync(0xFFFFFFFFu, fb);
      if (lane == 0) red[warp] = fb;
      __syncthreads();
      if (warp == 0) {
        uint32_t b = lane < nwarps ? red[lane] : 0xFFFFFFFFu;
        b = __reduce_min_sync(0xFFFFFFFFu, b);
        if (lane == 0) sh[0] = b;
      }
      __syncthreads();
      const uint32_t bit = sh[0];
      if (bit == 0xFFFFFFFFu) break;
      const uint32_t ib = stage * len + (bit >> 6);
      const uint64_t m = 1ull << (bit & 63);
      uint32_t cand = 0xFFFFFFFFu;
      for (uint32_t r = u + tid; r < rows; r += blockDim.x)
        if (xzs[(size_t)r * W + ib] & m) { cand = min(cand, r); break; }
      cand = __reduce_min_sync(0xFFFFFFFFu, cand);
      __syncthreads();
      if (lane == 0) red[warp] = cand;
      __syncthreads();
      if (warp == 0) {
        uint32_t b = lane < nwarps ? red[lane] : 0xFFFFFFFFu;
        b = __reduce_min_sync(0xFFFFFFFFu, b);
        if (lane == 0) sh[1] = b;
      }
      __syncthreads();
      const uint32_t c = sh[1];
      if (c == 0xFFFFFFFFu) { good = 0; break; }
      u = c + 1;
      if (tid == 0 && used && nu < cap) used[nu] = (int32_t)u;
      nu++;
      if (warp == 0) {
        uint64_t c1 = 0, c2 = 0;
        const uint64_t* l = xzs + (size_t)c * W;
        for (uint32_t w = lane; w < len; w += 32) {
          uint64_t x2 = p[w], z2 = p[len + w];
          mul_step_c(l[w], l[len + w], x2, z2, c1, c2);
          p[w] = x2;
          p[len + w] = z2;
        }
        if (phases) {
          const uint32_t s =
              __reduce_add_sync(0xFFFFFFFFu, (uint32_t)(__popcll(c1) + 2 * __popcll(c2)) & 3u) & 3u;
          if (lane == 0) sh[2] = (s + sh[2] + ph[c]) & 3u;
        }
      }
      __syncthreads();
    }
  }
  // the Pauli must now be the identity up to a phase
  uint32_t nz = 0;
  for (uint32_t w = tid; w < W; w += blockDim.x) nz |= p[w] != 0;
  nz = __reduce_or_sync(0xFFFFFFFFu, nz);
  if (lane == 0) red[warp] = nz;
  __syncthreads();
  if (tid == 0) {
    uint32_t any = 0;
    for (uint32_t k = 0; k < nwarps; k++) any |= red[k];
    ok[0] = (good && !any) ? 1 : 0;
    n_used[0] = nu;
    pph[0] = (uint8_t)sh[2];
  }
  for (uint32_t w = tid; w < W; w += blockDim.x) pauli[w] = p[w];
}

struct CanonPlan {
  uint32_t cs;
  bool smem_rows;
  size_t smem_bytes;
  uint32_t RB;
};

static size_t canon_smem(uint32_t rows, uint32_t W, uint32_t RB, bool smem_rows) {
  size_t b = (size_t)(W + 1) * 8;
  if (smem_rows) b += (size_t)RB * (W + 1) * 8;
  b += (2 + 32 + 4) * 4 + (size_t)rows * 4 + (size_t)RB * 4 + RB + 16;
  return (b + 15) / 16 * 16;
}

static uint32_t g_canon_cs = 0;       // tuner override (0 = automatic)
static uint32_t g_canon_threads = 0;  // tuner override (0 = automatic)

static CanonPlan canon_plan(uint32_t rows, uint32_t W) {
  const size_t maxsm = (size_t)device_max_smem_optin();
  if (g_canon_cs) {
    const uint32_t cs = g_canon_cs, RB = std::max<uint32_t>(1, (rows + cs - 1) / cs);
    const bool sm = canon_smem(rows, W, RB, true) <= maxsm;
    return {cs, sm, canon_smem(rows, W, RB, sm), RB};
  }
  // measured on B200 (random full-rank stabilizers, n = 1000 / 2000 / 4000):
  // 16 CTAs beat 8 / 4 / 2 / 1 at every size (3.4 / 8.8 / 47 ms); a small
  // tableau runs in one CTA with no cluster traffic
  const uint32_t big[] = {16, 8, 4, 2, 1}, small[] = {1, 2, 4, 8, 16};
  const uint32_t* cands = rows >= 256 ? big : small;
  for (uint32_t ci = 0; ci < 5; ci++) {
    const uint32_t cs = cands[ci];
    const uint32_t RB = std::max<uint32_t>(1, (rows + cs - 1) / cs);
    if (canon_smem(rows, W, RB, true) <= maxsm) return {cs, true, canon_smem(rows, W, RB, true), RB};
  }
  const uint32_t cs = 16, RB = std::max<uint32_t>(1, (rows + cs - 1) / cs);
  return {cs, false, canon_smem(rows, W, RB, false), RB};
}

int canonicalize_view(uint64_t* xzs, uint8_t* ph, uint32_t rows, uint32_t n, uint32_t W, int phases,
                      int32_t* d_out, cudaStream_t st) {
  if (rows == 0) {
    QCB_CUDA(cudaMemsetAsync(d_out, 0, 8, st));
    return QCB_OK;
  }
  CanonPlan p = canon_plan(rows, W);
  if (p.smem_bytes > (size_t)device_max_smem_optin())
    return fail(QCB_EUNSUPPORTED, "canonicalize!: tableau too tall for the cluster's bookkeeping");
  CanonArgs a{};
  a.xzs = xzs; a.ph = ph; a.rows = rows; a.n = n; a.W = W; a.RB = p.RB; a.phases = phases;
  a.smem_rows = p.smem_rows ? 1 : 0;
  a.out = d_out;
  if (!p.smem_rows) {
    QCB_CUDA(cudaMallocAsync(&a.gtmp, (size_t)rows * W * 8, st));
    QCB_CUDA(cudaMallocAsync(&a.gtmp_ph, rows, st));
  }
  QCB_CUDA(cudaFuncSetAttribute(canon_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_bytes));
  if (p.cs > 8) QCB_CUDA(cudaFuncSetAttribute(canon_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(p.cs);
  cfg.blockDim = dim3(g_canon_threads ? g_canon_threads : CANON_THREADS);
  cfg.dynamicSmemBytes = p.smem_bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  QCB_CUDA(cudaLaunchKernelEx(&cfg, canon_kernel, a));
  QCB_LAUNCHED();
  if (!p.smem_rows) {
    QCB_CUDA(cudaMemcpyAsync(xzs, a.gtmp, (size_t)rows * W * 8, cudaMemcpyDeviceToDevice, st));
    QCB_CUDA(cudaMemcpyAsync(ph, a.gtmp_ph, rows, cudaMemcpyDeviceToDevice, st));
    QCB_CUDA(cudaFreeAsync(a.gtmp, st));
    QCB_CUDA(cudaFreeAsync(a.gtmp_ph, st));
  }
  return QCB_OK;
}

int generate_dev(uint64_t* pauli, uint8_t* pph, const uint64_t* xzs, const uint8_t* ph, uint32_t rows,
                 uint32_t W, int phases, int32_t* d_ok, int32_t* d_used, uint32_t cap, uint32_t* d_nused,
                 cudaStream_t st) {
  const size_t sm = (size_t)W * 8;
  if (sm > 48 * 1024) QCB_CUDA(cudaFuncSetAttribute(generate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  generate_kernel<<<1, 1024, sm, st>>>(pauli, pph, xzs, ph, rows, W, phases, d_ok, d_used, cap, d_nused);
  QCB_LAUNCHED();
  return QCB_OK;
}

void set_canon_cluster(uint32_t cs) { g_canon_cs = cs; }
void set_canon_threads(uint32_t n) { g_canon_threads = n; }

}  // namespace qcb

using namespace qcb;

extern "C" {

int qcb_canonicalize(qcb_tableau* t, uint32_t row0, uint32_t nrows, int phases, int32_t* rx,
                     int32_t* rz, void* stream) {
  if (!t) return fail(QCB_EARG, "null tableau");
  if (row0 < 1 || (uint64_t)row0 - 1 + nrows > t->rows) return fail(QCB_EBOUNDS, "canonicalize!: row range out of bounds");
  cudaStream_t st = S(stream);
  int32_t* d_out = (int32_t*)t->scratch + 16;
  if (int s = canonicalize_view(t->xzs + (size_t)(row0 - 1) * t->W, t->phases + (row0 - 1), nrows,
                                t->nqubits, t->W, phases, d_out, st))
    return s;
  if (rx || rz) {
    int32_t h[2];
    QCB_CUDA(cudaMemcpyAsync(h, d_out, 8, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaStreamSynchronize(st));
    if (rx) *rx = h[0];
    if (rz) *rz = h[1];
  }
  return QCB_OK;
}

int qcb_generate(qcb_tableau* pauli, const qcb_tableau* stab, int phases, int32_t* ok, int32_t* used_rows,
                 uint32_t cap, uint32_t* n_used, void* stream) {
  if (!pauli || !stab || !ok) return fail(QCB_EARG, "null argument");
  if (pauli->nqubits != stab->nqubits) return fail(QCB_EDIM, "generate!: sizes differ");
  cudaStream_t st = S(stream);
  int32_t* d_ok = (int32_t*)pauli->scratch + 32;
  uint32_t* d_nu = (uint32_t*)pauli->scratch + 33;
  int32_t* d_used = nullptr;
  if (used_rows && cap) QCB_CUDA(cudaMallocAsync(&d_used, (size_t)cap * 4, st));
  if (int s = generate_dev(pauli->xzs, pauli->phases, stab->xzs, stab->phases, stab->rows, stab->W, phases,
                           d_ok, d_used, used_rows ? cap : 0, d_nu, st))
    return s;
  int32_t hok = 0;
  uint32_t hnu = 0;
  QCB_CUDA(cudaMemcpyAsync(&hok, d_ok, 4, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaMemcpyAsync(&hnu, d_nu, 4, cudaMemcpyDeviceToHost, st));
  QCB_CUDA(cudaStreamSynchronize(st));
  if (d_used) {
    QCB_CUDA(cudaMemcpyAsync(used_rows, d_used, (size_t)std::min(hnu, cap) * 4, cudaMemcpyDeviceToHost, st));
    QCB_CUDA(cudaFreeAsync(d_used, st));
    QCB_CUDA(cudaStreamSynchronize(st));
  }
  *ok = hok;
  if (n_used) *n_used = hnu;
  return QCB_OK;
}

}  // extern "C"
