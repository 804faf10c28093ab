// decode.cu -- the decoder hand-off of a sampled frame
// (src/ecc/decoder_pipeline.jl:163-193): the syndrome and fault columns of
// the record, the syndrome matrix a decoder consumes, and evaluate_guesses.
//
// The record lives as shot-packed bit planes (row b = record bit b, word c =
// shots 32c..32c+31).  A decoder wants it shot-major: per shot the selected
// bits in order.  `syndrome_rows_kernel` transposes 32 x 32 bit blocks with
// warp ballots (lane r holds row r's word; ballot of bit s over the lanes is
// shot s's 32 bits of those rows), stages a CTA's 32 shots in shared memory
// and writes them out contiguously.  `evaluate_guesses_kernel` works on
// planes: per 32 shots, the parity of the guessed faults selected by each
// row of the faults matrix against the measured logical row, a miss on any
// row failing the shot, then a popcount.
#include <algorithm>
#include <vector>

#include "qcb_internal.h"

namespace qcb {

// out[s, k] (column-major Bool, S x nsel) = record[rows[k], s] ^ flip[k].
__global__ void record_columns_kernel(const uint32_t* rec, uint64_t pitch, uint64_t S, const uint32_t* rows,
                                      const uint8_t* flip, uint32_t nsel, uint8_t* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // 4 shots per thread
  const uint32_t k = blockIdx.y;
  const uint64_t f = i * 4;
  if (f >= S || k >= nsel) return;
  const uint32_t word = __ldg(rec + (uint64_t)rows[k] * pitch + (f >> 5));
  const uint32_t sh = (uint32_t)(f & 31);
  const uint8_t x = flip ? (flip[k] & 1u) : 0u;
  uint8_t* dst = out + (uint64_t)k * S + f;
  for (uint32_t j = 0; j < 4 && f + j < S; j++) dst[j] = (uint8_t)(((word >> (sh + j)) & 1u) ^ x);
}

// Shot-major syndrome matrix: out[s * Wsyn + w] bit b = record[rows[64w + b], s]
// (bits past nsel are zero).  One CTA per 32 shots; warp g handles 64-row
// groups g, g + nwarps, ...; `stage` keeps the CTA's 32 x Wsyn words so the
// write-out is contiguous (stage == 0: direct writes).
__global__ void syndrome_rows_kernel(const uint32_t* rec, uint64_t pitch, uint64_t S, const uint32_t* rows,
                                     uint32_t nsel, uint32_t Wsyn, uint64_t* out, int stage) {
  extern __shared__ __align__(16) uint64_t tile[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint64_t c = blockIdx.x;  // word column: shots 32c .. 32c+31
  const uint64_t shot = c * 32 + lane;
  for (uint32_t g = warp; g < Wsyn; g += nw) {
    uint64_t v = 0;
    for (uint32_t half = 0; half < 2; half++) {
      const uint32_t r = g * 64 + half * 32 + lane;
      const uint32_t word = r < nsel ? __ldg(rec + (uint64_t)rows[r] * pitch + c) : 0u;
      uint32_t mine = 0;
#pragma unroll
      for (uint32_t s = 0; s < 32; s++) {
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, (word >> s) & 1u);
        if (s == lane) mine = b;
      }
      v |= (uint64_t)mine << (32 * half);
    }
    if (stage) tile[(size_t)lane * Wsyn + g] = v;
    else if (shot < S) out[shot * Wsyn + g] = v;
  }
  if (!stage) return;
  __syncthreads();
  const uint64_t s0 = c * 32;
  const uint32_t nshots = (uint32_t)(S - s0 < 32 ? S - s0 : 32);
  const uint32_t total = nshots * Wsyn;
  for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) out[s0 * Wsyn + t] = tile[t];
}

// guesses (column-major Bool S x k) -> planes [k][ncols] u32.
__global__ void bools_to_planes_kernel(const uint8_t* g, uint64_t S, uint32_t k, uint64_t ncols, uint32_t* planes) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t col = blockIdx.y;
  if (c >= ncols || col >= k) return;
  const uint8_t* src = g + (uint64_t)col * S + c * 32;
  uint32_t w = 0;
  const uint32_t n = (uint32_t)(S - c * 32 < 32 ? S - c * 32 : 32);
  for (uint32_t b = 0; b < n; b++) w |= (uint32_t)(src[b] & 1u) << b;
  planes[(uint64_t)col * ncols + c] = w;
}

// evaluate_guesses (src/ecc/decoder_pipeline.jl:172-190) over 32 shots per
// thread: shot s fails when some row j of the faults matrix gives
// parity(F[j,:] . guess_s) != measured fault j of shot s.  F is nlog rows of
// Fw 32-bit words in shared memory.
__global__ void evaluate_guesses_kernel(const uint32_t* rec, uint64_t pitch, uint64_t S, const uint32_t* log_rows,
                                        uint32_t nlog, const uint32_t* gplanes, uint32_t k, uint64_t ncols,
                                        const uint32_t* F, uint32_t Fw, unsigned long long* fails) {
  extern __shared__ uint32_t Fs[];
  for (uint32_t t = threadIdx.x; t < nlog * Fw; t += blockDim.x) Fs[t] = F[t];
  __syncthreads();
  uint32_t cnt = 0;
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bad = 0;
    for (uint32_t j = 0; j < nlog; j++) {
      uint32_t par = __ldg(rec + (uint64_t)log_rows[j] * pitch + c);
      for (uint32_t fw = 0; fw < Fw; fw++) {
        uint32_t m = Fs[j * Fw + fw];
        while (m) {
          const uint32_t b = __ffs(m) - 1;
          m &= m - 1;
          par ^= __ldg(gplanes + (uint64_t)(fw * 32 + b) * ncols + c);
        }
      }
      bad |= par;
    }
    const uint64_t base = c * 32;
    if (S - base < 32) bad &= (1u << (uint32_t)(S - base)) - 1u;
    cnt += __popc(bad);
  }
  cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(fails, (unsigned long long)cnt);
}

}  // namespace qcb

using namespace qcb;

// Validated 0-based record rows of 1-based bits.
static int record_rows(const qcb_frame* f, const uint32_t* bits, size_t n, std::vector<uint32_t>& rows) {
  rows.resize(n);
  for (size_t k = 0; k < n; k++) {
    if (bits[k] == 0) return fail(QCB_EZEROQUBIT, "record bits start at 1");
    if (bits[k] > f->nbits) return fail(QCB_EBOUNDS, "record bit exceeds the frame's measurements");
    rows[k] = bits[k] - 1;
  }
  return QCB_OK;
}

extern "C" {

int qcb_frame_measurement_columns(const qcb_frame* f, const uint32_t* bits, size_t nsel, const uint8_t* reference,
                                  uint8_t* bools, void* stream) {
  if (!f || (nsel && (!bits || !bools))) return fail(QCB_EARG, "null argument");
  std::vector<uint32_t> rows;
  if (int s = record_rows(f, bits, nsel, rows)) return s;
  if (!nsel || !f->frames) return QCB_OK;
  if (nsel > 65535) return fail(QCB_EARG, "at most 65535 columns per call");
  cudaStream_t st = S(stream);
  uint32_t* d_rows = nullptr;
  uint8_t *d_flip = nullptr, *d_out = nullptr;
  const size_t bytes = (size_t)f->frames * nsel;
  QCB_CUDA(cudaMallocAsync(&d_rows, nsel * 4, st));
  QCB_CUDA(cudaMallocAsync(&d_out, bytes, st));
  QCB_CUDA(cudaMemcpyAsync(d_rows, rows.data(), nsel * 4, cudaMemcpyHostToDevice, st));
  std::vector<uint8_t> flip;
  if (reference) {
    // measurements(register, frame): the Register's reference bits XORed in
    flip.resize(nsel);
    for (size_t k = 0; k < nsel; k++) flip[k] = reference[rows[k]] & 1u;
    QCB_CUDA(cudaMallocAsync(&d_flip, nsel, st));
    QCB_CUDA(cudaMemcpyAsync(d_flip, flip.data(), nsel, cudaMemcpyHostToDevice, st));
  }
  dim3 grid((unsigned)(((f->frames + 3) / 4 + 255) / 256), (unsigned)nsel);
  record_columns_kernel<<<grid, 256, 0, st>>>(f->record, f->pitch, f->frames, d_rows, d_flip, (uint32_t)nsel, d_out);
  QCB_LAUNCHED();
  QCB_CUDA(cudaMemcpyAsync(bools, d_out, bytes, cudaMemcpyDeviceToHost, st));
  cudaFreeAsync(d_rows, st);
  cudaFreeAsync(d_out, st);
  if (d_flip) cudaFreeAsync(d_flip, st);
  QCB_CUDA(cudaStreamSynchronize(st));
  return QCB_OK;
}

int qcb_frame_syndrome_rows(const qcb_frame* f, const uint32_t* bits, size_t nsel, uint64_t* out, int out_on_device,
                            void* stream) {
  if (!f || (nsel && (!bits || !out))) return fail(QCB_EARG, "null argument");
  std::vector<uint32_t> rows;
  if (int s = record_rows(f, bits, nsel, rows)) return s;
  if (!nsel || !f->frames) return QCB_OK;
  cudaStream_t st = S(stream);
  const uint32_t Wsyn = (uint32_t)((nsel + 63) / 64);
  const size_t out_bytes = (size_t)f->frames * Wsyn * 8;
  uint32_t* d_rows = nullptr;
  uint64_t* d_out = out;
  QCB_CUDA(cudaMallocAsync(&d_rows, nsel * 4, st));
  QCB_CUDA(cudaMemcpyAsync(d_rows, rows.data(), nsel * 4, cudaMemcpyHostToDevice, st));
  if (!out_on_device) QCB_CUDA(cudaMallocAsync(&d_out, out_bytes, st));
  const size_t sm = (size_t)32 * Wsyn * 8;
  const int stage = sm <= 48 * 1024 ? 1 : 0;
  syndrome_rows_kernel<<<(unsigned)f->ncols, 256, stage ? sm : 0, st>>>(f->record, f->pitch, f->frames, d_rows,
                                                                         (uint32_t)nsel, Wsyn, d_out, stage);
  QCB_LAUNCHED();
  if (!out_on_device) {
    QCB_CUDA(cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d_out, st);
  }
  cudaFreeAsync(d_rows, st);
  QCB_CUDA(cudaStreamSynchronize(st));  // rows lives on this stack frame
  return QCB_OK;
}

int qcb_evaluate_guesses(const qcb_frame* f, const uint32_t* logical_bits, size_t nlog, const uint8_t* guesses,
                         size_t k, const uint8_t* faults, uint64_t* fails, void* stream) {
  if (!f || !fails || (nlog && !logical_bits) || (k && (!guesses || !faults))) return fail(QCB_EARG, "null argument");
  std::vector<uint32_t> rows;
  if (int s = record_rows(f, logical_bits, nlog, rows)) return s;
  *fails = 0;
  if (!nlog || !f->frames) return QCB_OK;
  if (k > 65535) return fail(QCB_EARG, "at most 65535 guess columns");
  cudaStream_t st = S(stream);
  // faults: nlog x k Bool, column-major (Julia Matrix layout) -> bit rows
  const uint32_t Fw = (uint32_t)((k + 31) / 32);
  std::vector<uint32_t> F((size_t)nlog * std::max<uint32_t>(Fw, 1), 0);
  for (size_t j = 0; j < nlog; j++)
    for (size_t c = 0; c < k; c++)
      if (faults[c * nlog + j] & 1u) F[j * Fw + c / 32] |= 1u << (c % 32);
  const size_t smF = F.size() * 4;
  if (smF > 200 * 1024) return fail(QCB_EARG, "faults matrix too large for one call");
  uint32_t *d_rows = nullptr, *d_F = nullptr, *d_planes = nullptr;
  uint8_t* d_g = nullptr;
  unsigned long long* d_fails = nullptr;
  QCB_CUDA(cudaMallocAsync(&d_rows, nlog * 4, st));
  QCB_CUDA(cudaMallocAsync(&d_F, smF, st));
  QCB_CUDA(cudaMallocAsync(&d_fails, 8, st));
  QCB_CUDA(cudaMemcpyAsync(d_rows, rows.data(), nlog * 4, cudaMemcpyHostToDevice, st));
  QCB_CUDA(cudaMemcpyAsync(d_F, F.data(), smF, cudaMemcpyHostToDevice, st));
  QCB_CUDA(cudaMemsetAsync(d_fails, 0, 8, st));
  if (k) {
    QCB_CUDA(cudaMallocAsync(&d_g, (size_t)f->frames * k, st));
    QCB_CUDA(cudaMallocAsync(&d_planes, (size_t)k * f->ncols * 4, st));
    QCB_CUDA(cudaMemcpyAsync(d_g, guesses, (size_t)f->frames * k, cudaMemcpyHostToDevice, st));
    dim3 g1((unsigned)((f->ncols + 255) / 256), (unsigned)k);
    bools_to_planes_kernel<<<g1, 256, 0, st>>>(d_g, f->frames, (uint32_t)k, f->ncols, d_planes);
    QCB_LAUNCHED();
  }
  if (smF > 48 * 1024)
    QCB_CUDA(cudaFuncSetAttribute(evaluate_guesses_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smF));
  const uint32_t blocks = (uint32_t)std::min<uint64_t>((f->ncols + 255) / 256, 4ull * device_sm_count());
  evaluate_guesses_kernel<<<std::max<uint32_t>(blocks, 1), 256, smF, st>>>(
      f->record, f->pitch, f->frames, d_rows, (uint32_t)nlog, d_planes, (uint32_t)k, f->ncols, d_F, Fw, d_fails);
  QCB_LAUNCHED();
  unsigned long long h = 0;
  QCB_CUDA(cudaMemcpyAsync(&h, d_fails, 8, cudaMemcpyDeviceToHost, st));
  cudaFreeAsync(d_rows, st);
  cudaFreeAsync(d_F, st);
  cudaFreeAsync(d_fails, st);
  if (d_g) cudaFreeAsync(d_g, st);
  if (d_planes) cudaFreeAsync(d_planes, st);
  QCB_CUDA(cudaStreamSynchronize(st));
  *fails = h;
  return QCB_OK;
}

}  // extern "C"
