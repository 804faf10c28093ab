// qcb_internal.h -- shared internals of libqcb200 (host + device).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <string>
#include <vector>

#include "../../include/qcb200.h"

namespace qcb {

// ------------------------------------------------------------ errors
void set_error(int status, const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
extern std::atomic<uint64_t> g_launches;

#define QCB_CUDA(call)                                        \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::qcb::cuda_fail(e_, #call); \
  } while (0)

// Check the launch that was just issued and count it.
#define QCB_LAUNCHED()                                                 \
  do {                                                                 \
    ::qcb::g_launches.fetch_add(1, std::memory_order_relaxed);         \
    cudaError_t e_ = cudaGetLastError();                               \
    if (e_ != cudaSuccess) return ::qcb::cuda_fail(e_, "kernel launch"); \
  } while (0)

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

int device_sm_count();
int device_max_smem_optin();

// ------------------------------------------------------------ Philox
enum : uint32_t { TAG_INITZ = 0x51A7u, TAG_RESET = 0x5E5Eu, TAG_NOISE = 0x4E01u };

// Philox-4x32-10 (Salmon et al., SC'11), published multipliers and Weyl
// increments.  Counter = (index, column lo, column hi, tag), key = seed.
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                       uint32_t c3, uint32_t k0, uint32_t k1,
                                                       uint32_t out[4]) {
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int r = 0; r < 10; r++) {
#ifdef __CUDA_ARCH__
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// ------------------------------------------------------------ programs
// Device program: a stream of 16-byte records.  Operands are physical plane
// indices of the frame tile (plane 2s / 2s+1 of slot s, swapped while the
// qubit is relabelled by an odd number of x<->z gates).
//   header (4 words): [kind<<24 | count, aux0, aux1, aux2], then operands.
enum SegKind : uint32_t {
  SEG_END = 0,
  SEG_CNOT = 1,   // count entries (x_c, z_c, x_t, z_t)
  SEG_H = 2,      // compile-time only (relabel); never emitted
  SEG_S = 3,      // entries (x, z, opcode, 0): z ^= x
  SEG_G1 = 4,     // entries (x, z, opcode, 0)
  SEG_G2 = 5,     // entries (opcode, x_a, z_a, x_b), (z_b, 0, 0, 0)
  SEG_MZ = 6,     // entries (x, bit), padded to a multiple of 4 words
  SEG_MRZ = 7,    // count groups of 4 entries (x, z, bit or NONE, reset or PAD)
  SEG_FLUSH = 8,  // count sites (site, kind | class << 8, x_a | z_a << 16, x_b | z_b << 16)
  SEG_CZ = 9,     // entries (x_a, z_a, x_b, z_b)
  SEG_WIN = 10,   // the stream continues in the next window
  SEG_XOR = 11    // entries of 32 words (store, n, b_0 .. b_{n-1}, 0 ...): record row
                  // store <- XOR of record rows b_i (ClassicalXOR)
};
// Inputs of one ClassicalXOR entry.
constexpr uint32_t XOR_MAX_BITS = 30;
// Entry layouts in the windowed stream (planes are 16-bit):
//   CNOT/CZ (x_a | z_a<<16, x_b | z_b<<16); S/G1 (x | z<<16, opcode);
//   G2 (x_a | z_a<<16, x_b | z_b<<16, opcode, 0); MZ (x, bit);
//   MRZ groups of 4 x (x | z<<16, bit, reset or PAD, 0); FLUSH as above.
// Header word 1 bit 0: no barrier after this record (a record split across
// windows; its parts are independent).
constexpr uint32_t BIT_NONE = 0xFFFFFFFFu;
constexpr uint32_t MRZ_PAD = 0xFFFFFFFFu;
constexpr uint32_t FLAG_NO_BARRIER = 1u;
// FLUSH header word 1: bit 1 = the part has dense sites (drawn in the walk),
// bits 8.. = the part's pre-sampler bucket capacity; word 2 = the part index,
// word 3 = the bucket's offset in a group's events.
constexpr uint32_t FLAG_DENSE_SITES = 2u;
// Program window staged into shared memory by the walker (words).
constexpr uint32_t PROG_WINDOW_WORDS = 2048;      // program window (8 KB)
constexpr uint32_t PROG_WINDOW_WORDS_TALL = 4096; // tall programs with records longer than 8 KB (16 KB)

// Sampling parameters shared by the noise sites of one opcode with equal
// probabilities, in fixed point so that the device does integer work only.
//  dense  (one 32-bit word w per shot): PauliNoise X if w < thr0, Z if
//         w < thr1, Y if w < thr2; Depolarization an event if w < thr2, of
//         Pauli index 1 + w*np/thr2.  Thresholds in units of 2^-32.
//  sparse (one word per group gives the event count k: the first k with
//         w < cdf[cdf_off + k], else cdf_len; each event is one word w with
//         position w & (NOISE_GROUP-1) and kind word v = w >> 10):
//         PauliNoise X if v < thr0, Z if v < thr1, else Y; Depolarization
//         Pauli index 1 + (v*np >> 22).  Thresholds in units of 2^-22.
struct NoiseClass {
  uint64_t thr0, thr1, thr2;
  uint32_t dense, np, cdf_off, cdf_len;
};
// Longest Binomial count table (counts above it are clamped to it; sparse
// classes have NOISE_GROUP*p_eff <= NOISE_DENSE_LAMBDA, so the clamped tail
// has probability below 2^-60).
constexpr uint32_t NOISE_CDF_MAX = 128;
constexpr uint32_t NOISE_KIND_BITS = 22;
// Noise is sampled per (site, group of NOISE_GROUP consecutive shots).
constexpr uint32_t NOISE_GROUP = 1024;
// Sites with p_eff * NOISE_GROUP above this draw every shot (dense mode).
constexpr double NOISE_DENSE_LAMBDA = 16.0;

// A noise site: kind = opcode (PAULI_NOISE / DEPOL1 / DEPOL2), the planes of
// its qubit(s) at the noise op, the total event probability p_eff and the
// thresholds for the event kind, and the Binomial(NOISE_GROUP, p_eff)
// parameters of the event count: q0 = (1-p_eff)^NOISE_GROUP, r = p_eff/(1-p_eff).
struct Site {
  uint32_t kind, xa, za, xb;
  uint32_t zb, dense, pad0, pad1;
  double t0, t1, t2;  // PAULI: X if v<t0, Z if v<t1, Y if v<t2
  double peff, q0, r;
};

struct Program {
  qcb_program_info info;
  uint32_t nq;         // qubits referenced (max index)
  uint32_t nslots;     // distinct qubits referenced (smem slots); scratch = nslots
  std::vector<uint32_t> slot_qubit;   // slot -> 0-based qubit
  std::vector<uint32_t> stream_slot;  // operands in slot space; scratch slot = nslots
  uint32_t win_words = PROG_WINDOW_WORDS;  // words per window of stream_slot
  std::vector<Site> sites_slot;
  std::vector<int64_t> site_of_op;    // op index -> site (or -1)
  std::vector<uint32_t> site_arity;
  std::vector<uint8_t> slot_swap;     // final x<->z relabel per slot
  std::vector<NoiseClass> classes;
  std::vector<uint32_t> cdf;          // Binomial count thresholds of the sparse classes
  double pmax = 0;
  // Pre-sampling of the sparse noise sites (a kernel that draws every (site,
  // group) before the walk): one entry per sparse site of a flush part,
  // (site, kind | class << 8, part j, entry index i in the part); per part
  // the bucket capacity (events per group), cumulative in pre_capoff.
  std::vector<uint4> pre_ent;
  std::vector<uint32_t> pre_capoff;   // [nparts + 1]
  uint32_t pre_nparts = 0;
  // device copies
  uint32_t* d_stream_slot = nullptr;
  NoiseClass* d_classes = nullptr;
  uint32_t* d_cdf = nullptr;
  uint32_t* d_slot_qubit = nullptr;
  uint32_t* d_slot_swap = nullptr;
  uint32_t* d_qubit_slot = nullptr;   // [nq_alloc] qubit -> slot or NONE
  uint4* d_pre_ent = nullptr;
  uint32_t* d_pre_capoff = nullptr;
  uint32_t qubit_slot_len = 0;
  uint64_t hash = 0;
};

}  // namespace qcb

struct qcb_program : qcb::Program {};

struct qcb_frame {
  uint64_t frames;
  uint32_t qubits;   // user qubits (frame has qubits+1)
  uint32_t nq1;      // qubits + 1
  uint32_t nbits;
  uint64_t ncols;    // ceil(frames/32)
  uint64_t pitch;    // words per plane (>= ncols, multiple of 32)
  uint32_t* planes;  // [(2*(nq1+1))][pitch]: plane 2q = x(q), 2q+1 = z(q); last pair = scratch
  uint32_t* record;  // [nbits][pitch]
  int32_t* err;      // device status word of the walker (QCB_ETIMEOUT on a stuck wait)
  // scratch of the noise pre-sampler (event buckets and counters), grown on
  // demand; only frames made by qcb_frame_create own one (pre_own)
  uint32_t* pre = nullptr;
  uint64_t pre_bytes = 0;
  bool pre_own = false;
};

namespace qcb {
int run_chunk(qcb_frame* f, uint64_t ncols, const qcb_program* p, uint64_t seed, uint64_t shot_offset, uint32_t* rec,
              uint64_t rec_pitch, cudaStream_t st);
// Tile width and CTAs of the walker launch that run_chunk makes for `ncols`
// columns of program p.
void chunk_shape(const qcb_program* p, uint64_t ncols, uint32_t* tile, uint32_t* ctas);
// Bytes of noise pre-sampler scratch a chunk of `ncols` columns of program p
// needs (0: the program has no pre-sampled noise); a chunk frame that holds at
// least that much at `pre` (pre_own false) gets its noise pre-sampled, any
// other chunk draws it in the walk.
uint64_t chunk_presample_bytes(const qcb_program* p, uint64_t ncols);
}  // namespace qcb

struct qcb_tableau {
  uint32_t rows;
  uint32_t nqubits;
  uint32_t W;        // words per row = 2*ceil(n/64)
  uint64_t* xzs;     // rows x W, row-contiguous
  uint8_t* phases;   // rows
  uint32_t* scratch; // small device scratch (phase accumulators, flags)
};
