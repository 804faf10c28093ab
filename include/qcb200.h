/*
 * qcb200.h -- C ABI of libqcb200, a B200-native (sm_100a) implementation of the
 * bit-packed tableau / Pauli-frame hot path of QuantumClifford.jl v0.11.7.
 *
 * The library replaces the device methods that the reference's CUDA package
 * extension supplies (the files of ext/QuantumCliffordGPUExt) and the KernelAbstractions
 * `mul_left!` (ext/QuantumCliffordKAExt/mul_leftright.jl).  A Julia extension
 * binds these symbols with `ccall`; every signature uses plain pointers, sizes
 * and POD structs only.
 *
 * Conventions
 *  - Qubit and record-bit indices inside qcb_op are 1-based, exactly as in the
 *    Julia operation structs (sCNOT(1,2), sMZ(3,1), ...).  A record bit of 0
 *    means "do not record" (reference: sMZ(q) / sMRZ(q) with bit 0).
 *  - Row indices passed to tableau calls are 1-based (Julia convention).
 *  - Every call returns an int status (QCB_OK == 0).  qcb_last_error() gives
 *    the message of the last failing call on the calling host thread.
 *  - Calls are asynchronous on the given stream (NULL = the legacy default
 *    stream), except calls that return host values (phases, ranks, projection
 *    results), which synchronise that stream before returning.
 *  - Host buffers are borrowed for the duration of the call only; all device
 *    memory is owned by the library behind opaque handles.
 */
#ifndef QCB200_H
#define QCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum qcb_status {
  QCB_OK = 0,
  QCB_EDIM = 1,        /* DimensionMismatch (src/throws.jl:8-14)                 */
  QCB_EBOUNDS = 2,     /* BoundsError: qubit / bit / row index out of range       */
  QCB_EZEROQUBIT = 3,  /* ArgumentError(NoZeroQubit) (src/throws.jl:1)           */
  QCB_EARG = 4,        /* ArgumentError, e.g. two-qubit gate with q1 == q2
                          (src/symbolic_cliffords.jl:351)                        */
  QCB_EOOM = 5,        /* device allocation failed                               */
  QCB_EBUDGET = 6,     /* request exceeds the configured HBM budget              */
  QCB_ETIMEOUT = 7,    /* a device-side bounded wait expired                     */
  QCB_ECUDA = 8,       /* CUDA runtime error                                     */
  QCB_EBADSTRUCT = 9,  /* BadDataStructure (src/project_trace_reset.jl:352-354)  */
  QCB_EUNSUPPORTED = 10,
  QCB_ENOTREADY = 11   /* asynchronous result not yet available                  */
};

/* ------------------------------------------------------------------ ops   */
/* Operation codes.  Gate truth tables follow src/symbolic_cliffords.jl
 * (`@qubitop1` at :105-118, `@qubitop2` at :358-395).                       */
enum qcb_opcode {
  QCB_OP_NOP = 0,
  /* single-qubit symbolic Cliffords */
  QCB_OP_I = 1, QCB_OP_H = 2, QCB_OP_S = 3, QCB_OP_SDAG = 4,
  QCB_OP_X = 5, QCB_OP_Y = 6, QCB_OP_Z = 7,
  QCB_OP_SQRTX = 8, QCB_OP_INVSQRTX = 9, QCB_OP_SQRTY = 10, QCB_OP_INVSQRTY = 11,
  QCB_OP_HXY = 12, QCB_OP_HYZ = 13, QCB_OP_CXYZ = 14, QCB_OP_CZYX = 15,
  /* SingleQubitOperator(q1, xx, xz, zx, zz, px, pz) (src/symbolic_cliffords.jl
   * :168-206): its flags packed in q2, bit 0 xx, 1 xz, 2 zx, 3 zz, 4 px, 5 pz.
   * x' = (x & xx) ^ (z & zx), z' = (x & xz) ^ (z & zz).                      */
  QCB_OP_SQO = 16,
  /* two-qubit symbolic Cliffords */
  QCB_OP_CNOT = 32, QCB_OP_CPHASE = 33, QCB_OP_SWAP = 34,
  QCB_OP_ZCX = 35, QCB_OP_ZCY = 36, QCB_OP_ZCZ = 37,
  QCB_OP_XCX = 38, QCB_OP_XCY = 39, QCB_OP_XCZ = 40,
  QCB_OP_YCX = 41, QCB_OP_YCY = 42, QCB_OP_YCZ = 43,
  QCB_OP_SWAPCX = 44, QCB_OP_INVSWAPCX = 45, QCB_OP_ISWAP = 46, QCB_OP_INVISWAP = 47,
  QCB_OP_CZSWAP = 48, QCB_OP_CXSWAP = 49, QCB_OP_ZCRY = 50, QCB_OP_INVZCRY = 51,
  QCB_OP_SQRTZZ = 52, QCB_OP_INVSQRTZZ = 53, QCB_OP_SQRTXX = 54, QCB_OP_INVSQRTXX = 55,
  QCB_OP_SQRTYY = 56, QCB_OP_INVSQRTYY = 57,
  QCB_OP_LAST2Q = 57,  /* two-qubit gates are QCB_OP_CNOT..QCB_OP_LAST2Q */
  /* measurements (frame semantics: src/pauli_frames.jl:74-116) */
  QCB_OP_MZ = 64, QCB_OP_MRZ = 65, QCB_OP_MX = 66, QCB_OP_MRX = 67,
  /* ClassicalXOR(bits, store) (src/misc_ops.jl:198-205; frame semantics
   * src/pauli_frames.jl:63-72): record bit `bit` <- XOR of n = q1 record bits
   * (1 <= n <= 30), which follow in the next ceil(n/3) ops of opcode
   * QCB_OP_XOR_BITS, three 1-based bits each in q1, q2, bit (0 = none).      */
  QCB_OP_XOR = 68, QCB_OP_XOR_BITS = 69,
  /* noise */
  QCB_OP_PAULI_NOISE = 96, /* PauliError(q, px, py, pz): NoiseOp(PauliNoise)   */
  QCB_OP_DEPOL1 = 97,      /* NoiseOp(DepolarizationNoise(p), (q1,))           */
  QCB_OP_DEPOL2 = 98       /* NoiseOp(DepolarizationNoise(p), (q1, q2))        */
};

/* One circuit operation (40 bytes, 8-byte aligned).
 *  - q1, q2: 1-based qubits (q2 only for two-qubit gates and DEPOL2).
 *  - bit:    1-based record bit for MZ/MRZ/MX/MRX; 0 = not recorded.
 *  - p:      PAULI_NOISE: p[0]=px, p[1]=py, p[2]=pz  (src/noise.jl:56-60);
 *            DEPOL1/DEPOL2: p[0] = depolarisation probability p as in
 *            DepolarizationNoise(p) (src/noise.jl:34-53): with probability p a
 *            uniformly random k-qubit Pauli, identity included, is applied.  */
typedef struct qcb_op {
  uint32_t opcode;
  uint32_t q1;
  uint32_t q2;
  uint32_t bit;
  double p[3];
} qcb_op;

/* Where the randomness of a frame run comes from. */
enum qcb_noise_mode {
  QCB_NOISE_PHILOX = 0, /* on-device Philox-4x32-10 per site and shot group   */
  QCB_NOISE_MASK = 1    /* caller-supplied events (bit-exact parity mode)      */
};

/* A noise event for mask mode: at noise op `op_index` (0-based index into
 * the op array given to qcb_program_compile), frame `shot` (0-based) suffers
 * Pauli `pauli`.  PAULI_NOISE: 1 = X, 2 = Z, 3 = Y.  DEPOL1/DEPOL2: the index
 * of the Pauli in base 4, first qubit least significant, digits 0=I 1=X 2=Z
 * 3=Y (src/noise.jl:99-129).                                                */
typedef struct qcb_event {
  uint32_t op_index;
  uint32_t pauli;
  uint64_t shot;
} qcb_event;

typedef struct qcb_noise_source {
  uint32_t mode;         /* qcb_noise_mode                                   */
  uint32_t reserved;
  uint64_t seed;         /* PHILOX: key                                      */
  uint64_t shot_offset;  /* global index of this frame's shot 0; a multiple
                            of 32.  Shards of one run use disjoint offsets.  */
  /* MASK mode only (host pointers, borrowed for the call): */
  const qcb_event* events;
  uint64_t n_events;
  /* One bit plane per MRZ/MRX op in program order: plane k, word w, bit b is
   * the `rand(Bool)` of that reset for shot 32*w+b (src/pauli_frames.jl:112).
   * Shape [n_resets][ceil(frames/32)] uint32.  NULL = all zero.            */
  const uint32_t* reset_planes;
} qcb_noise_source;

typedef struct qcb_program_info {
  uint32_t nqubits;       /* highest qubit used                             */
  uint32_t nbits;         /* highest record bit used                        */
  uint32_t n_ops;         /* ops given                                      */
  uint32_t n_updates;     /* Clifford + measurement ops per frame           */
  uint32_t n_noise_sites; /* noise sites (one per qubit of PauliError)      */
  uint32_t n_resets;      /* MRZ/MRX ops                                    */
  uint32_t n_segments;    /* fused segments in the device program           */
  uint32_t n_flushes;     /* noise flush points                             */
} qcb_program_info;

typedef struct qcb_program qcb_program;
typedef struct qcb_frame qcb_frame;
typedef struct qcb_tableau qcb_tableau;

/* ------------------------------------------------------------ library     */
/* Select the device and create its context.  Also raises the release
 * threshold of the device's default stream-ordered memory pool to at least
 * 1 GB, so that the per-call scratch of the tableau calls stays in the pool
 * between calls instead of being mapped through the driver each time.      */
int qcb_init(int device);
const char* qcb_version(void);
int qcb_last_error(char* buf, size_t len);
const char* qcb_status_string(int status);
int qcb_device_synchronize(void);
/* Count of this library's kernel launches since load (for launch accounting). */
uint64_t qcb_launch_count(void);

/* ------------------------------------------------------------ programs    */
/* Compile a circuit into a device program (replaces the per-op dispatch of
 * pftrajectories(frame, circuit), src/pauli_frames.jl:234-239, and
 * compactify_circuit, src/sumtypes.jl:190-237).  Validates indices like the
 * Julia constructors do.                                                    */
int qcb_program_compile(const qcb_op* ops, size_t n_ops, qcb_program** out);
int qcb_program_info_get(const qcb_program* prog, qcb_program_info* info);
/* Bytes of the program that the walker reads from device memory (records,
 * noise classes, Binomial count tables): what qcb_pftrajectories_host copies
 * host -> device on each call.  No reference counterpart (a size query). */
int qcb_program_device_bytes(const qcb_program* prog, uint64_t* bytes);
int qcb_program_destroy(qcb_program* prog);

/* ------------------------------------------------------------ Pauli frames */
/* PauliFrame(frames, qubits, measurements) (src/pauli_frames.jl:30-37): an
 * (qubits+1)-qubit frame (hidden ancilla included), zero x/z bits, an
 * all-false record of `nbits` bits.  initZ! is a separate call.             */
int qcb_frame_create(uint64_t frames, uint32_t qubits, uint32_t nbits, qcb_frame** out);
int qcb_frame_destroy(qcb_frame* f);
int qcb_frame_shape(const qcb_frame* f, uint64_t* frames, uint32_t* qubits, uint32_t* nbits);
/* initZ! (src/pauli_frames.jl:47-56) from Philox (seed, shot_offset).       */
int qcb_frame_init_z(qcb_frame* f, uint64_t seed, uint64_t shot_offset, void* stream);
/* initZ! from caller bit planes [qubits+1][ceil(frames/32)] (mask mode).   */
int qcb_frame_init_z_planes(qcb_frame* f, const uint32_t* z_planes, void* stream);
/* Zero the x/z bits and the record.                                        */
int qcb_frame_clear(qcb_frame* f, void* stream);
/* copy(frame) (src/pauli_frames.jl:17): dst <- src, planes and record, on
 * the device; both frames have the same shape (QCB_EDIM otherwise).        */
int qcb_frame_copy(qcb_frame* dst, const qcb_frame* src, void* stream);

/* pftrajectories(frame, circuit) (src/pauli_frames.jl:234-239).            */
int qcb_pftrajectories(qcb_frame* f, const qcb_program* prog,
                       const qcb_noise_source* noise, void* stream);

/* apply!(frame, op) for a short op list (compiled on the fly).             */
int qcb_frame_apply_ops(qcb_frame* f, const qcb_op* ops, size_t n_ops,
                        const qcb_noise_source* noise, void* stream);

/* Reference-layout transfers.  `xzs` is the parent of the Adjoint matrix of
 * a fastcolumn frame: frames x W' uint64, frames contiguous per word, with
 * W' = 2*ceil((qubits+1)/64) (X words first, then Z words;
 * src/fastmemlayout.jl:45-60, src/pauli_frames.jl:30-37).  Padding bits are
 * written as zero.                                                          */
int qcb_frame_download_xzs(const qcb_frame* f, uint64_t* xzs, void* stream);
int qcb_frame_upload_xzs(qcb_frame* f, const uint64_t* xzs, void* stream);
/* measurements(frame) (src/pauli_frames.jl:280): Bool matrix frames x nbits,
 * column-major (one byte per bit).                                         */
int qcb_frame_download_measurements(const qcb_frame* f, uint8_t* bools, void* stream);
/* The record from a reference frame's Bool matrix (frames x nbits,
 * column-major, nonzero = true): PauliFrame(frame, measurements) moved to the
 * device (the measurements field of src/pauli_frames.jl:9-12).             */
int qcb_frame_upload_measurements(qcb_frame* f, const uint8_t* bools, void* stream);
/* The record as shot-packed bit planes [nbits][ceil(frames/32)] uint32.    */
int qcb_frame_download_record_planes(const qcb_frame* f, uint32_t* planes, void* stream);
/* x/z planes [qubits+1][ceil(frames/32)] uint32 each (device layout).      */
int qcb_frame_download_planes(const qcb_frame* f, uint32_t* x_planes, uint32_t* z_planes, void* stream);

/* ------------------------------------------------------------ batches
 * Many sampling jobs drained from one persistent launch (no reference
 * counterpart: the reference runs one pftrajectories per circuit).  Each job
 * is a fresh run (initZ! + circuit, Philox mode) of `program` on `frame`, so
 * its record equals that of qcb_pftrajectories_fresh with the same seed and
 * shot_offset.  The (job, shot-tile) items are queued longest first and taken
 * by one CTA per SM.  qcb_batch_run only clears the queue head and launches:
 * it can be captured in a CUDA graph.  Frames and programs must outlive the
 * batch; the frame tile of every job must fit one CTA's shared memory.      */
typedef struct qcb_batch_job {
  qcb_frame* frame;
  const qcb_program* program;
  uint64_t seed;
  uint64_t shot_offset;   /* a multiple of 1024                                */
  uint32_t tile;          /* shot columns per tile (even, 16..256); 0 = tuned
                             width of the job's size class, else the widest  */
  uint32_t reserved;
} qcb_batch_job;
typedef struct qcb_batch qcb_batch;
int qcb_batch_create(const qcb_batch_job* jobs, size_t n_jobs, qcb_batch** out);
int qcb_batch_run(qcb_batch* b, void* stream);
/* Synchronising check of every job's device status word (QCB_ETIMEOUT when a
 * device-side wait expired).                                                */
int qcb_batch_status(const qcb_batch* b);
int qcb_batch_destroy(qcb_batch* b);
/* The autotuner: times the candidate tile widths (16..256 columns) for
 * `program` on a scratch frame of two full waves each and records the fastest
 * per frame column for the program's size class (its touched qubits), which
 * qcb_batch_create then uses.  Synchronises the device.                     */
int qcb_tune_tile(const qcb_program* program, uint32_t* tile, float* us_per_column, void* stream);
/* The plain walker's autotuner: times `program` on a scratch frame of
 * `frames` shots for the tile widths (the cost model's choice and the
 * power-of-two widths that fit shared memory) and 448 / 512 / 576 / 640
 * threads per CTA, and records the fastest pair for the program's size class
 * (its touched qubits) at that frame width: later fresh runs of exactly that
 * width take it (results are identical for any launch shape).  Returns the
 * pair and its time per run.  Synchronises the device.
 * qcb_tune_walker_clear forgets every recorded pair.                       */
int qcb_tune_walker(const qcb_program* program, uint64_t frames, uint32_t* tile, uint32_t* threads,
                    float* ms, void* stream);
int qcb_tune_walker_clear(void);

/* ------------------------------------------------------------ serving
 * A request loop with continuous batching (no reference counterpart).
 * Requests (an op list, shots, seed) are submitted at any time from any host
 * thread; their programs are compiled once per distinct op list and stay
 * resident.  A scheduler thread admits requests first come, first served as
 * a slot (a CUDA stream), the HBM budget (the full record plus one shot
 * chunk's frame planes from a pool) and the GPU's fill allow (the running
 * requests' remaining walker CTAs leave SMs idle: small requests and the
 * last chunk of a large one share the GPU, large ones run in arrival order),
 * and runs each as a sequence of fresh Philox shot chunks of `chunk_shots`
 * (0 = 2^20), two in flight; every record equals that of one plain run of
 * the request (qcb_pftrajectories_fresh, same seed, shot_offset 0).
 * Records stay on the device until qcb_server_release.                   */
typedef struct qcb_server qcb_server;
int qcb_server_create(uint64_t hbm_budget_bytes, uint32_t slots, uint64_t chunk_shots, qcb_server** out);
int qcb_server_submit(qcb_server* s, const qcb_op* ops, size_t n_ops, uint64_t shots, uint64_t seed,
                      uint64_t* ticket);
/* Compile an op list into the resident program cache without running it.  */
int qcb_server_preload(qcb_server* s, const qcb_op* ops, size_t n_ops);
/* state: 0 queued, 1 running, 2 done, 3 failed (the status is then the
 * request's error); times3 (may be NULL): submit, admit and completion
 * times in seconds since the server started.                               */
int qcb_server_query(qcb_server* s, uint64_t ticket, int32_t* state, double* times3);
int qcb_server_wait(qcb_server* s, uint64_t ticket, double timeout_s);
/* The next request that finished or failed and was not reported yet, in
 * completion order (blocks up to timeout_s; QCB_ETIMEOUT when none did).    */
int qcb_server_next_done(qcb_server* s, double timeout_s, uint64_t* ticket, int32_t* state, double* times3);
/* The record of a finished request: nbits x ceil(shots/32) uint32 planes
 * (host memory; may be NULL to read *nbits only).                          */
int qcb_server_result(qcb_server* s, uint64_t ticket, uint32_t* planes, uint32_t* nbits);
int qcb_server_release(qcb_server* s, uint64_t ticket);
/* Device bytes charged to the budget (records, chunk planes and resident
 * programs), of which the resident programs, and their number.  No
 * reference counterpart (the reference has no server).                     */
int qcb_server_stats(qcb_server* s, uint64_t* used_bytes, uint64_t* program_bytes, uint32_t* n_programs);
int qcb_server_destroy(qcb_server* s);

/* The decoder hand-off (src/ecc/decoder_pipeline.jl:163-170).
 * measurements(frame)[:, bits]: the record columns `bits` (1-based, nsel of
 * them) as a Bool matrix S x nsel, column-major (the reference's view of the
 * syndrome or logical bits).  `reference` (nbits Bools, may be NULL) is
 * XORed in: measurements(register, frame) (src/pauli_frames.jl:289).       */
int qcb_frame_measurement_columns(const qcb_frame* f, const uint32_t* bits, size_t nsel,
                                  const uint8_t* reference, uint8_t* bools, void* stream);
/* The syndrome matrix for a decoder, shot-major and bit-packed: shot s owns
 * words out[s*W .. s*W+W-1], W = ceil(nsel/64), bit b of word w = record bit
 * bits[64w+b] of shot s (zero past nsel).  out is device memory when
 * out_on_device, else host memory (the call then synchronises).           */
int qcb_frame_syndrome_rows(const qcb_frame* f, const uint32_t* bits, size_t nsel, uint64_t* out,
                            int out_on_device, void* stream);
/* evaluate_guesses(measured_faults, guesses, faults_matrix)
 * (src/ecc/decoder_pipeline.jl:172-190) with measured_faults =
 * measurements(frame)[:, logical_bits]: guesses is the decoder's Bool matrix
 * S x k and faults the Bool matrix nlog x k, both column-major (host);
 * *fails gets the number of failed shots (the reference returns
 * fails / nsamples).                                                       */
int qcb_evaluate_guesses(const qcb_frame* f, const uint32_t* logical_bits, size_t nlog,
                         const uint8_t* guesses, size_t k, const uint8_t* faults, uint64_t* fails,
                         void* stream);

/* pftrajectories(circuit; trajectories) (src/pauli_frames.jl:193-227) as one
 * host call: fresh frame, Philox initZ!, run, record copied back as
 * shot-packed planes [nbits][ceil(frames/32)]; returns when the record is
 * in `record_planes` (NULL: run only).  The op list is compiled on the host
 * when it differs from the last call's; the compiled program (records,
 * noise classes, count tables: qcb_program_device_bytes) is copied host ->
 * device from page-locked memory on every call.  The device buffers of the
 * program and of the frame of the last shape are kept (on the device current
 * at the first call) for reuse.  Wide runs go as shot chunks whose
 * record columns are copied out while the next chunk runs; the record is
 * that of one launch.  Page-locked `record_planes` gets the full PCIe
 * bandwidth.  Calls are serialised by an internal lock.                     */
int qcb_pftrajectories_host(const qcb_op* ops, size_t n_ops, uint64_t frames,
                            uint64_t seed, uint64_t shot_offset,
                            uint32_t* record_planes, void* stream);

/* pftrajectories(circuit; trajectories) on a preallocated frame: initZ!
 * (Philox, seed / shot_offset) fused with the run; x starts at zero.  The
 * record keeps the previous contents of bits the program does not write.   */
int qcb_pftrajectories_fresh(qcb_frame* f, const qcb_program* prog, uint64_t seed,
                             uint64_t shot_offset, void* stream);

/* Launch-shape overrides used by the tuner ("walker_tile", "canon_threads",
 * "canon_cluster", "project_cluster", "canon_blocked": 1 always / 2 never
 * run canonicalize! by 64-column panels); 0 restores the automatic choice.
 * Test knob "stage_withhold" k > 0: the plain walker never stages window k of
 * each CTA's program windows, so its bounded wait expires and the run reports
 * QCB_ETIMEOUT at the next synchronising call (the kernel returns; nothing
 * faults); a fresh run or initZ! of the frame clears that status.  Test
 * knob "server_hash_bits" b > 0: the serving program cache keeps only b low
 * bits of its hash, so distinct circuits collide (the byte comparison on a
 * hit keeps results right).  Knob "server_fill" (read by qcb_server_create):
 * 1 (default) admits onto idle SMs only, 0 whenever a slot is free.
 * canonicalize! by panels over the whole GPU: "canon_grid" 0 (automatic:
 * stabilizer views of 640..8192 rows) / 1 always / 2 never; "canon_rpt"
 * rows per pivot-search thread (0: automatic, 1, 2, 4, 8, 16);
 * "canon_apply_rows" rows per apply CTA (0 or 8..32); "canon_pdl" 1
 * (default) / 0: the panel launches as programmatic dependent launches or
 * plain; "canon_lookahead" 1 (default) / 0: each panel's pivot steps run
 * beside the previous panel's grid-wide apply, or the two in turn.  project! on the whole GPU: "project_grid" 0 (automatic: generic
 * Paulis on Stabilizer kinds too tall for one cluster's shared memory) / 1
 * always where it applies / 2 never.  Test knob "project_withhold" 1: one CTA
 * of that kernel leaves before the first grid barrier, the others' bounded
 * waits expire and the call returns QCB_ETIMEOUT (nothing faults).  Noise:
 * "presample" 0 (automatic) / 1 never (draw in the walk) / 2 every bucket
 * overflows (test).  "walker_threads" threads per walker CTA (0: 640, or
 * 64..640 in steps of 32); "walker_pdl" 1 (default) / 0: the walker as a
 * programmatic dependent launch of the noise pre-sampler or plain;
 * "walker_narrow" 1 (default) / 0: programs too tall for a 16-column
 * shared-memory tile run in 8..14-column tiles, or on the HBM planes.
 * "gates_pdl" 1 (default) / 0: qcb_apply_gates launches as programmatic
 * dependents of the launch before them on the stream, or plain.            */
int qcb_tune_set(const char* key, int64_t value);

/* ------------------------------------------------------------ tableaux    */
/* A Tableau in the reference layout (src/QuantumClifford.jl:145-151): `rows`
 * Pauli rows over `nqubits`; row r is W = 2*ceil(nqubits/64) uint64 words,
 * X words then Z words; phases are uint8 mod 4.  A PauliOperator is a
 * one-row tableau.                                                          */
int qcb_tableau_create(uint32_t rows, uint32_t nqubits, qcb_tableau** out);
int qcb_tableau_destroy(qcb_tableau* t);
int qcb_tableau_shape(const qcb_tableau* t, uint32_t* rows, uint32_t* nqubits);
int qcb_tableau_upload(qcb_tableau* t, const uint8_t* phases, const uint64_t* xzs, void* stream);
int qcb_tableau_download(const qcb_tableau* t, uint8_t* phases, uint64_t* xzs, void* stream);
int qcb_tableau_copy(qcb_tableau* dst, const qcb_tableau* src, void* stream);

/* mul_left!(r::PauliOperator, l::PauliOperator; phases)
 * (src/mul_leftright.jl:137-142, 75-126): r <- l * r.  r and l are one-row
 * tableaux of equal size.  The new phase of r is written to *phase_out
 * (may be NULL).                                                            */
int qcb_mul_left_pauli(qcb_tableau* r, const qcb_tableau* l, int phases,
                       uint8_t* phase_out, void* stream);
/* No counterpart in the reference.  Batched mul_left! (the semantics of
 * qcb_mul_left_pauli) on caller-owned device memory, allocating nothing:
 * for i < count, Pauli r_i <- l_i * r_i, where pair i is row i of two
 * count-row tableaux in the reference layout (r_xz + i*W, W =
 * 2*ceil(nqubits/64) uint64 words, X words then Z words; phases uint8,
 * updated in place when `phases` is nonzero, left untouched otherwise).
 * For callers that hold their Paulis in memory of another allocator and call
 * from a loop where a device allocation (and the device-wide synchronisation
 * a free implies) is not acceptable.  The phase accumulators live in one
 * static device array of QCB_NOALLOC_MAX_PAIRS words per device: count above
 * it fails with QCB_EARG.  The array starts at zero and every call leaves it
 * at zero.  The first call on a device looks the array up
 * (cudaGetSymbolAddress, with that device current) and clears it, so make it
 * before any latency-critical use.  Calls that overlap in time on one device
 * (other streams or host threads) share the array and race: serialise them.
 * The array's address is kept per device for the life of the process: after
 * a cudaDeviceReset (or a reset of the primary context) of a device, do not
 * call this entry point on that device again in the same process.          */
#define QCB_NOALLOC_MAX_PAIRS 4096
int qcb_mul_left_pauli_batch_noalloc(uint64_t* r_xz, uint8_t* r_phases, const uint64_t* l_xz,
                                     const uint8_t* l_phases, uint32_t nqubits, uint32_t count,
                                     int phases, void* stream);
/* rowswap!(state, i, j; phases) (src/QuantumClifford.jl:899-927): rows i, j
 * (1-based) of the state's stabilizer view; the Destabilizer kinds swap the
 * paired destabilizer rows too; phases move only when `phases`.           */
int qcb_rowswap(qcb_tableau* t, int kind, uint32_t i, uint32_t j, int phases, void* stream);
/* mul_left!(s::Tableau, m, i; phases) (src/mul_leftright.jl:177-181).      */
int qcb_mul_left_row(qcb_tableau* s, uint32_t m, uint32_t i, int phases, void* stream);
/* The mul_left! / mul_right! family on rows (src/mul_leftright.jl:137-245;
 * the device methods of ext/QuantumCliffordKAExt/mul_leftright.jl:101-460).
 * For k < count, target row a = s_row + k of s and source row
 * b = t_row + k * t_step of t (1-based; t_step 0 repeats one source row):
 *   right == 0: s[a] <- t[b] * s[a]    (mul_left!)
 *   right != 0: s[a] <- s[a] * t[b]    (mul_right!)
 * With `phases`, s.phases[a] <- (extra + s.phases[a] + P) & 3, where P is
 * t.phases[b] (phase_src 0: the PauliOperator forms, mul_left!(s, p), and the
 * KA extension's methods) or s.phases[b] (phase_src 1: the reference's
 * mul_left!(s, m, t, i) / mul_right!(s, m, t, i), which read s.phases[i],
 * src/mul_leftright.jl:171-175, 183-187).  s and t may be one tableau; then
 * the source rows must not overlap the target rows (unless they are the same
 * rows, count > 1).  With count == 1 and phase_out non-NULL the new phase is
 * written there (the call then synchronises the stream).                    */
int qcb_mul_rows(qcb_tableau* s, uint32_t s_row, uint32_t count, const qcb_tableau* t, uint32_t t_row,
                 uint32_t t_step, int right, int phase_src, int phases, uint8_t* phase_out, void* stream);
/* mul_left!(state, i, j; phases) (src/mul_leftright.jl:194-219), 1-based:
 * Stabilizer / MixedStabilizer: row i <- row j * row i of the tableau;
 * Destabilizer / MixedDestabilizer (2n rows): destabilizer j <- destabilizer
 * i * destabilizer j without phases, then stabilizer i <- stabilizer j *
 * stabilizer i (rows n+i, n+j) with phases.                                 */
int qcb_mul_left_state(qcb_tableau* s, int kind, uint32_t i, uint32_t j, int phases, void* stream);
/* mul_left!(s::Tableau, p::PauliOperator; phases) (src/mul_leftright.jl:223-229). */
int qcb_mul_left_tableau_pauli(qcb_tableau* s, const qcb_tableau* p, int phases, void* stream);
/* prodphase / comm of row i of l and row j of r (src/QuantumClifford.jl:723-859). */
int qcb_prodphase(const qcb_tableau* l, uint32_t i, const qcb_tableau* r, uint32_t j,
                  uint8_t* out, void* stream);
int qcb_comm(const qcb_tableau* l, uint32_t i, const qcb_tableau* r, uint32_t j,
             uint8_t* out, void* stream);

/* canonicalize!(state; phases, ranks) (src/canonicalization.jl:92-133) on rows
 * [row0, row0+nrows) of t (1-based row0; the stabilizer view).  rx, rz get
 * the last pivot indices of the X and Z stage (relative to the view), as
 * with ranks=true.                                                          */
int qcb_canonicalize(qcb_tableau* t, uint32_t row0, uint32_t nrows, int phases,
                     int32_t* rx, int32_t* rz, void* stream);

/* Tableau kinds for project!. */
enum qcb_state_kind {
  QCB_STABILIZER = 0,         /* rows = the stabilizer                       */
  QCB_MIXED_STABILIZER = 1,   /* rows >= rank; *rank_io = rank               */
  QCB_DESTABILIZER = 2,       /* rows = 2n' (destabilizers then stabilizers) */
  QCB_MIXED_DESTABILIZER = 3  /* rows = 2*nqubits; *rank_io = rank           */
};

/* project!(state, pauli; keep_result, phases) (src/project_trace_reset.jl:231-439).
 * `paulis` holds k one-row Paulis (a k-row tableau); they are projected in
 * order on the same state.  anticom[j] gets the anticommuting index (0 if
 * none); result[j] gets the measurement phase 0..3, or -1 for `nothing`.
 * For the mixed kinds *rank_io is read and updated.  A status of
 * QCB_EBADSTRUCT reports BadDataStructure for projection j = *n_done.       */
int qcb_project(qcb_tableau* t, int kind, int32_t* rank_io, const qcb_tableau* paulis,
                int keep_result, int phases, int32_t* anticom, int32_t* result,
                uint32_t* n_done, void* stream);

/* projectX!(state, qubit) / projectZ! / projectY! (src/project_trace_reset.jl
 * :440-573): k single-qubit projections in order, basis 1 = X, 2 = Z, 3 = Y,
 * qubits 1-based.  On a MixedDestabilizer this is project_cond! (a one-bit
 * anticommutation test per row; the new stabilizer row is the projector with
 * phase 0); on the other kinds project! with single_x/z/y, as the reference
 * dispatches.  Outputs as for qcb_project.                                  */
int qcb_project_qubit(qcb_tableau* t, int kind, int32_t* rank_io, uint32_t basis,
                      const uint32_t* qubits, size_t k, int keep_result, int phases,
                      int32_t* anticom, int32_t* result, uint32_t* n_done, void* stream);

/* projectrand!(state, pauli) / projectXrand! / projectZrand! / projectYrand!
 * (src/project_trace_reset.jl:575-636): the projections of qcb_project (when
 * `paulis` is non-NULL) or of qcb_project_qubit (basis, qubits, k), with
 * keep_result and phases on; a projection whose outcome is undetermined
 * (`nothing`) sets the new stabilizer row's phase to rand_phases[j] (0 or 2,
 * drawn by the caller, one per projection) and reports it as the result.    */
int qcb_projectrand(qcb_tableau* t, int kind, int32_t* rank_io, const qcb_tableau* paulis,
                    uint32_t basis, const uint32_t* qubits, size_t k, const uint8_t* rand_phases,
                    int32_t* anticom, int32_t* result, uint32_t* n_done, void* stream);

/* canonicalize!(state; phases, ranks) (src/canonicalization.jl:92-133) on a
 * whole state of the given kind (rank for the mixed kinds): for Destabilizer
 * and MixedDestabilizer the row swaps and products also act on the paired
 * destabilizer rows, as rowswap!/mul_left! on those states do
 * (src/QuantumClifford.jl:907-927, src/mul_leftright.jl:200-219).          */
int qcb_canonicalize_state(qcb_tableau* t, int kind, int32_t rank, int phases,
                           int32_t* rx, int32_t* rz, void* stream);

/* canonicalize_rref!(state, colindices; phases) (src/canonicalization.jl
 * :150-185): cols are 1-based qubits in order; *i_out gets the reference's
 * returned index i (1-based; rows i+1.. hold the pivots).                   */
int qcb_canonicalize_rref(qcb_tableau* t, int kind, int32_t rank, const uint32_t* cols,
                          size_t ncols, int phases, int32_t* i_out, void* stream);

/* canonicalize_gott!(stabilizer; phases) (src/canonicalization.jl:206-272)
 * without backtracking: r, s and the permutations xperm, zperm (1-based,
 * nqubits entries each, may be NULL) that were applied with permutesystems!. */
int qcb_canonicalize_gott(qcb_tableau* t, int phases, int32_t* r, int32_t* s,
                          uint32_t* xperm, uint32_t* zperm, void* stream);

/* permutesystems!(s, perm) (src/linalg.jl:7-17): every row becomes row[perm]
 * (new qubit j is old qubit perm[j], 1-based, nqubits entries); phases stay. */
int qcb_permutesystems(qcb_tableau* t, const uint32_t* perm, void* stream);

/* Many canonicalize! jobs on Stabilizer tableaux drained by persistent
 * thread-block clusters (no reference counterpart), each job exactly
 * qcb_canonicalize on that tableau.  cluster: CTAs per cluster for every job
 * (0 = one CTA per job running by 64-column panels, its rows in global memory
 * when they do not fit; tableaux outside 64..4096 rows by column steps on the
 * smallest cluster that holds them).  Jobs of one kind and cluster size form
 * a class, one persistent launch per class on its own stream, forked from and
 * joined back to `stream`.  run launches only
 * (capturable in a CUDA graph); ranks synchronises the device and gives each
 * job's rx, rz in the caller's order.  The tableaux must outlive the batch. */
typedef struct qcb_canon_batch qcb_canon_batch;
int qcb_canon_batch_create(qcb_tableau* const* tabs, size_t n, int phases, uint32_t cluster,
                           qcb_canon_batch** out);
int qcb_canon_batch_run(qcb_canon_batch* b, void* stream);
int qcb_canon_batch_ranks(const qcb_canon_batch* b, int32_t* rx, int32_t* rz);
int qcb_canon_batch_destroy(qcb_canon_batch* b);

/* expect(p, s) (src/project_trace_reset.jl:743-751) for each of the k
 * one-row Paulis in `paulis` on the state `t` of the given kind (rank for the
 * mixed kinds), each on its own copy, in one launch; `t` is not modified.
 * out[j] = -1 for 0 (the reference's `nothing`), else the phase q of the
 * result i^q: 0 -> 1, 1 -> im, 2 -> -1, 3 -> -im.                          */
int qcb_expect(const qcb_tableau* t, int kind, int32_t rank, const qcb_tableau* paulis, int32_t* out,
               void* stream);

/* generate!(pauli, stabilizer; phases) (src/project_trace_reset.jl:37-81) on
 * a canonical stabilizer.  Writes the remaining Pauli (identity up to phase)
 * back into `pauli`; *ok = 0 when the Pauli cannot be generated.  used_rows
 * (capacity cap, may be NULL) gets the 1-based rows used, *n_used their count. */
int qcb_generate(qcb_tableau* pauli, const qcb_tableau* stab, int phases, int32_t* ok,
                 int32_t* used_rows, uint32_t cap, uint32_t* n_used, void* stream);

/* apply!(state, gates) for symbolic gates with phases
 * (src/symbolic_cliffords.jl:62-74, 293-316), applied in order.  Each launch
 * (up to 128 gates) is a programmatic dependent of the launch before it on
 * the stream, so a stream of single-gate calls overlaps each launch with the
 * previous kernel; the kernel reads the rows only once its predecessor has
 * completed, so the order of calls on the stream is kept.                   */
int qcb_apply_gates(qcb_tableau* t, const qcb_op* ops, size_t n_ops, int phases, void* stream);

/* Dense apply!(state, c::CliffordOperator; phases) (src/dense_cliffords.jl:135-169).
 * `c` is the 2n-row tableau of the Clifford operator (images of X_1..X_n,
 * then Z_1..Z_n).                                                           */
int qcb_apply_dense(qcb_tableau* t, const qcb_tableau* c, int phases, void* stream);

/* ------------------------------------------------------------ diagnostics */
/* Philox-4x32-10 block (counter, key) -> out, computed on the device.       */
int qcb_debug_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Compile on the host only (no device needed) and copy out the device
 * program: the record stream (uint32 words), the noise-site table (80 bytes
 * per site), and per slot the frame qubit and the final x<->z relabel flag.
 * Buffers may be NULL or too small, in which case only the sizes are set.   */
int qcb_debug_program_dump(const qcb_op* ops, size_t n_ops, uint32_t* stream, size_t stream_cap,
                           size_t* stream_len, uint8_t* sites, size_t sites_cap, size_t* n_sites,
                           uint32_t* slot_qubit, uint32_t* slot_swap, size_t slots_cap, size_t* n_slots,
                           qcb_program_info* info);

#ifdef __cplusplus
}
#endif
#endif /* QCB200_H */
