# QuantumCliffordB200Ext -- Julia package extension that routes QuantumClifford's
# bit-packed tableau / Pauli-frame hot path to libqcb200 (B200, sm_100a) through
# `ccall`.  It plays the role ext/QuantumCliffordGPUExt plays for CUDA.jl
# arrays (ext/QuantumCliffordGPUExt/types.jl:22-53): the reference's own types
# -- Tableau, Stabilizer, Destabilizer, MixedStabilizer, MixedDestabilizer,
# PauliOperator, PauliFrame -- hold device storage types defined here
# (B200Matrix, B200Phases, B200Planes, B200Record, ...), and methods are
# selected by dispatch on that storage, so user code keeps calling
# pftrajectories, measurements, apply!, mul_left!, canonicalize!, project! ...
#
#   f = to_b200(PauliFrame(10^6, n, nbits))    # PauliFrame{Stabilizer{Tableau{B200FramePhases,B200Planes}},B200Record}
#   pftrajectories(f, circuit)                 # one launch (program compiled once per circuit content)
#   m = measurements(f)                        # Matrix{Bool}, as the reference returns
#   s = to_b200(random_stabilizer(1000))       # Stabilizer{Tableau{B200Phases,B200Matrix}}
#   canonicalize!(s); project!(s, to_b200(random_pauli(1000)))
#   frames = pftrajectories(on_b200(circuit); trajectories=10^6)   # pftrajectories(circuit; trajectories)
#   ECC.evaluate_decoder(decoder, nsamples, on_b200(circuit), syndrome_bits, logical_bits, faults)
#
# The extension needs two stubs in QuantumClifford (next to to_gpu/to_cpu in
# src/gpu_adapters.jl): `function to_b200 end` and `function on_b200 end`.
# Not exercised in this repository (no Julia toolchain here); the same C ABI
# is exercised by the Python mirror in ../qcb200 and its tests.
module QuantumCliffordB200Ext

using LinearAlgebra: Adjoint
using QuantumClifford
using QuantumClifford: AbstractOperation, AbstractSymbolicOperator, AbstractSingleQubitOperator,
    AbstractTwoQubitOperator, NoiseOp, NoisyGate, NoiseOpAll, PauliNoise, UnbiasedUncorrelatedNoise,
    DepolarizationNoise, affectedqubits, affectedbits, SingleQubitOperator, ClassicalXOR, PauliMeasurement,
    CliffordOperator, PauliFrame, Tableau, ECC
import QuantumClifford: apply!, pftrajectories, measurements, initZ!, applynoise!, mul_left!, mul_right!,
    canonicalize!, canonicalize_rref!, canonicalize_gott!, permutesystems!, project!, projectX!, projectY!,
    projectZ!, projectXrand!, projectYrand!, projectZrand!, expect, generate!, rowswap!, prodphase, comm,
    nqubits, to_cpu, to_b200, on_b200

const libqcb = get(ENV, "QCB200_LIB", joinpath(@__DIR__, "..", "lib", "libqcb200.so"))

# ---------------------------------------------------------------- errors
function _check(st::Cint)
    st == 0 && return nothing
    buf = Vector{UInt8}(undef, 4096)
    ccall((:qcb_last_error, libqcb), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
    msg = unsafe_string(pointer(buf))
    st == 1 && throw(DimensionMismatch(msg))                     # src/throws.jl:8-14
    st == 2 && throw(BoundsError(msg))
    (st == 3 || st == 4) && throw(ArgumentError(msg))            # NoZeroQubit, q1 == q2
    st == 9 && throw(QuantumClifford.BadDataStructure(msg, :project!, :Destabilizer))
    error("libqcb200 status $st: $msg")
end

_b(::Val{B}) where {B} = B
_b(x::Bool) = x

_noscalar() = throw(ArgumentError("scalar indexing of B200 device storage; move the object with to_cpu first"))

# ---------------------------------------------------------------- ops
struct QcbOp            # mirrors `qcb_op` (40 bytes)
    opcode::UInt32
    q1::UInt32
    q2::UInt32
    bit::UInt32
    p::NTuple{3,Float64}
end

const OPC = Dict{DataType,UInt32}(
    sId1 => 1, sHadamard => 2, sPhase => 3, sInvPhase => 4, sX => 5, sY => 6, sZ => 7,
    sSQRTX => 8, sInvSQRTX => 9, sSQRTY => 10, sInvSQRTY => 11, sHadamardXY => 12, sHadamardYZ => 13,
    sCXYZ => 14, sCZYX => 15, sCNOT => 32, sCPHASE => 33, sSWAP => 34, sZCX => 35, sZCY => 36,
    sZCZ => 37, sXCX => 38, sXCY => 39, sXCZ => 40, sYCX => 41, sYCY => 42, sYCZ => 43,
    sSWAPCX => 44, sInvSWAPCX => 45, sISWAP => 46, sInvISWAP => 47, sCZSWAP => 48, sCXSWAP => 49,
    sZCrY => 50, sInvZCrY => 51, sSQRTZZ => 52, sInvSQRTZZ => 53, sSQRTXX => 54, sInvSQRTXX => 55,
    sSQRTYY => 56, sInvSQRTYY => 57,
    sMZ => 64, sMRZ => 65, sMX => 66, sMRX => 67)

_qcbops(op::AbstractSingleQubitOperator) = [QcbOp(OPC[typeof(op)], op.q, 0, 0, (0.0, 0.0, 0.0))]
_qcbops(op::AbstractTwoQubitOperator) = [QcbOp(OPC[typeof(op)], op.q1, op.q2, 0, (0.0, 0.0, 0.0))]
_qcbops(op::Union{sMZ,sMRZ,sMX,sMRX}) = [QcbOp(OPC[typeof(op)], op.qubit, 0, op.bit, (0.0, 0.0, 0.0))]
# SingleQubitOperator: opcode 16, the six Bool fields as flag bits 0..5 of q2
_qcbops(op::SingleQubitOperator) = [QcbOp(16, op.q, op.xx | op.xz << 1 | op.zx << 2 | op.zz << 3 | op.px << 4 | op.pz << 5,
                                          0, (0.0, 0.0, 0.0))]
# ClassicalXOR: one op 68 (q1 = number of bits, bit = store), then the bits three per op 69
function _qcbops(op::ClassicalXOR)
    b = collect(op.bits)
    ops = [QcbOp(68, length(b), 0, op.store, (0.0, 0.0, 0.0))]
    for i in 1:3:length(b)
        c = vcat(b[i:min(i + 2, end)], zeros(Int, 3))
        push!(ops, QcbOp(69, c[1], c[2], c[3], (0.0, 0.0, 0.0)))
    end
    ops
end
# PauliMeasurement on a frame (src/pauli_frames.jl:118-134): couple each
# qubit onto the ancilla n+1, then sMRZ(n+1, bit); the sign's sX does not
# change a frame
function _qcbops(op::PauliMeasurement)
    n = nqubits(op.pauli)
    ops = QcbOp[]
    for q in 1:n
        x, z = op.pauli[q]
        x && !z && push!(ops, QcbOp(40, q, n + 1, 0, (0.0, 0.0, 0.0)))
        !x && z && push!(ops, QcbOp(32, q, n + 1, 0, (0.0, 0.0, 0.0)))
        x && z && push!(ops, QcbOp(41, q, n + 1, 0, (0.0, 0.0, 0.0)))
    end
    push!(ops, QcbOp(65, n + 1, 0, op.bit, (0.0, 0.0, 0.0)))
    ops
end
function _qcbops(op::NoiseOp)
    n = op.noise
    if n isa UnbiasedUncorrelatedNoise
        return [QcbOp(96, q, 0, 0, (n.p / 3, n.p / 3, n.p / 3)) for q in op.indices]
    elseif n isa PauliNoise
        return [QcbOp(96, q, 0, 0, (n.px, n.py, n.pz)) for q in op.indices]
    elseif n isa DepolarizationNoise && length(op.indices) == 1
        return [QcbOp(97, op.indices[1], 0, 0, (n.p, 0.0, 0.0))]
    elseif n isa DepolarizationNoise && length(op.indices) == 2
        return [QcbOp(98, op.indices[1], op.indices[2], 0, (n.p, 0.0, 0.0))]
    end
    throw(ArgumentError("noise model $(typeof(n)) is not supported on the B200 path"))
end
# NoisyGate (src/noise.jl:178-190): the gate, then the noise on its qubits
_qcbops(op::NoisyGate) = vcat(_qcbops(op.gate), _qcbops(NoiseOp(op.noise, collect(affectedqubits(op.gate)))))
_qcbops(op, n::Integer) = _qcbops(op)
# NoiseOpAll (src/noise.jl:173-176, 192-195): the noise on qubits 1..n, n the
# frame's qubit count (the hidden ancilla excluded)
function _qcbops(op::NoiseOpAll, n::Integer)
    n >= 1 || throw(ArgumentError("NoiseOpAll needs the frame's qubit count (no qubit is known)"))
    _qcbops(NoiseOp(op.noise, collect(1:n)))
end
# A circuit, lowered for a frame of n qubits; n = 0 takes the highest qubit of
# the circuit's other ops (what pftrajectories(circuit; trajectories) sizes
# its frame by)
function _qcbops(circuit::AbstractVector, n::Integer=0)
    if n < 1
        n = maximum((op isa NoiseOpAll ? 0 : maximum(affectedqubits(op), init=0) for op in circuit), init=0)
    end
    reduce(vcat, (_qcbops(op, n) for op in circuit); init=QcbOp[])
end

struct NoiseSource   # mirrors `qcb_noise_source`
    mode::UInt32
    reserved::UInt32
    seed::UInt64
    shot_offset::UInt64
    events::Ptr{Cvoid}
    n_events::UInt64
    reset_planes::Ptr{UInt32}
end

# ---------------------------------------------------------------- programs
mutable struct B200Program
    handle::Ptr{Cvoid}
    function B200Program(ops::Vector{QcbOp})
        h = Ref{Ptr{Cvoid}}(C_NULL)
        _check(ccall((:qcb_program_compile, libqcb), Cint, (Ptr{QcbOp}, Csize_t, Ref{Ptr{Cvoid}}), ops, length(ops), h))
        p = new(h[])
        finalizer(x -> ccall((:qcb_program_destroy, libqcb), Cint, (Ptr{Cvoid},), x.handle), p)
    end
end

# Compiled programs keyed by the lowered op list itself (Dict compares the
# contents on a hash hit), so a circuit mutated in place compiles anew and an
# equal circuit built again hits; at most _MAX_PROGRAMS stay, least recently
# used dropped first (their device memory goes with the finalizer).
const _MAX_PROGRAMS = 64
const _programs = Dict{Vector{QcbOp},B200Program}()
const _program_lru = Vector{Vector{QcbOp}}()
function _program(ops::Vector{QcbOp})
    p = get(_programs, ops, nothing)
    if p === nothing
        p = B200Program(ops)
        _programs[copy(ops)] = p
        push!(_program_lru, copy(ops))
        while length(_program_lru) > _MAX_PROGRAMS
            delete!(_programs, popfirst!(_program_lru))
        end
    else
        i = findfirst(==(ops), _program_lru)
        i === nothing || push!(_program_lru, popat!(_program_lru, i))
    end
    p
end

# ---------------------------------------------------------------- frame storage
mutable struct FrameHandle         # owner of one qcb_frame
    ptr::Ptr{Cvoid}
    frames::Int
    qubits::Int                    # user qubits (the device frame has qubits + 1)
    nbits::Int
    seed::UInt64                   # Philox key of the next noisy call
end
function FrameHandle(frames::Integer, qubits::Integer, nbits::Integer, seed::UInt64)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _check(ccall((:qcb_frame_create, libqcb), Cint, (UInt64, UInt32, UInt32, Ref{Ptr{Cvoid}}), frames, qubits, nbits, h))
    f = FrameHandle(h[], frames, qubits, nbits, seed)
    finalizer(x -> ccall((:qcb_frame_destroy, libqcb), Cint, (Ptr{Cvoid},), x.ptr), f)
end

"""The frame bit planes on the device, seen as the `xzs` of a fastcolumn
frame tableau: (W', frames) UInt64, W' = 2*cld(qubits+1, 64)."""
struct B200Planes <: AbstractMatrix{UInt64}
    h::FrameHandle
end
Base.size(p::B200Planes) = (2 * cld(p.h.qubits + 1, 64), p.h.frames)
Base.getindex(::B200Planes, ::Int, ::Int) = _noscalar()

"""Frames track no phase (src/pauli_frames.jl:58-61): a zero phase per frame."""
struct B200FramePhases <: AbstractVector{UInt8}
    h::FrameHandle
end
Base.size(p::B200FramePhases) = (p.h.frames,)
Base.getindex(::B200FramePhases, ::Int) = 0x0

"""The measurement record on the device (shot-packed bit planes), seen as the
reference's frames x nbits Bool matrix."""
struct B200Record <: AbstractMatrix{Bool}
    h::FrameHandle
end
Base.size(r::B200Record) = (r.h.frames, r.h.nbits)
Base.getindex(::B200Record, ::Int, ::Int) = _noscalar()

const FrameTableauB200 = Tableau{B200FramePhases,B200Planes}
"""A PauliFrame whose frame and record live on the B200."""
const PauliFrameB200 = PauliFrame{Stabilizer{FrameTableauB200},B200Record}

_fh(f::PauliFrameB200) = f.measurements.h

function _frame_b200(frames::Integer, qubits::Integer, nbits::Integer; seed::UInt64=rand(UInt64))
    h = FrameHandle(frames, qubits, nbits, seed)
    PauliFrame(Stabilizer(Tableau(B200FramePhases(h), qubits + 1, B200Planes(h))), B200Record(h))
end

"""to_b200(frame::PauliFrame): the frame (x/z bits, reference fastcolumn or
fastrow layout) and its record moved to the device."""
function to_b200(f::PauliFrame; seed::Integer=rand(UInt64))
    g = _frame_b200(length(f), nqubits(f), size(f.measurements, 2); seed=UInt64(seed))
    xzs = f.frame.tab.xzs                        # (W', frames)
    host = xzs isa Adjoint ? Matrix{UInt64}(parent(xzs)) : Matrix{UInt64}(permutedims(xzs))
    _check(ccall((:qcb_frame_upload_xzs, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Ptr{Cvoid}), _fh(g).ptr, host, C_NULL))
    m = Matrix{Bool}(f.measurements)
    _check(ccall((:qcb_frame_upload_measurements, libqcb), Cint, (Ptr{Cvoid}, Ptr{Bool}, Ptr{Cvoid}), _fh(g).ptr, m, C_NULL))
    g
end

"""to_cpu(frame): the reference PauliFrame (fastcolumn frame, Bool record)."""
function to_cpu(f::PauliFrameB200)
    h = _fh(f)
    W = 2 * cld(h.qubits + 1, 64)
    xzs = Matrix{UInt64}(undef, h.frames, W)          # frames contiguous per word
    _check(ccall((:qcb_frame_download_xzs, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Ptr{Cvoid}), h.ptr, xzs, C_NULL))
    stab = Stabilizer(Tableau(zeros(UInt8, h.frames), h.qubits + 1, xzs'))   # fastcolumn: Adjoint storage
    PauliFrame(stab, measurements(f))
end

# initZ! (src/pauli_frames.jl:47-56) from Philox
function initZ!(f::PauliFrameB200)
    h = _fh(f)
    _check(ccall((:qcb_frame_init_z, libqcb), Cint, (Ptr{Cvoid}, UInt64, UInt64, Ptr{Cvoid}), h.ptr, h.seed, 0, C_NULL))
    h.seed += 0x9E3779B97F4A7C15
    f
end

# pftrajectories(frame, circuit) (src/pauli_frames.jl:234-239): the whole
# circuit in one launch, its program compiled once per circuit content
function pftrajectories(f::PauliFrameB200, circuit)
    h = _fh(f)
    src = Ref(NoiseSource(0, 0, h.seed, 0, C_NULL, 0, C_NULL))
    prog = _program(_qcbops(circuit, h.qubits))
    _check(ccall((:qcb_pftrajectories, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{NoiseSource}, Ptr{Cvoid}),
                 h.ptr, prog.handle, src, C_NULL))
    h.seed += 0x9E3779B97F4A7C15   # the next call draws fresh randomness
    f
end

# apply!(frame, op): a short op list compiled on the fly (no program cache)
function _apply_ops!(f::PauliFrameB200, ops::Vector{QcbOp})
    h = _fh(f)
    src = Ref(NoiseSource(0, 0, h.seed, 0, C_NULL, 0, C_NULL))
    _check(ccall((:qcb_frame_apply_ops, libqcb), Cint, (Ptr{Cvoid}, Ptr{QcbOp}, Csize_t, Ref{NoiseSource}, Ptr{Cvoid}),
                 h.ptr, ops, length(ops), src, C_NULL))
    h.seed += 0x9E3779B97F4A7C15
    f
end
apply!(f::PauliFrameB200, op::AbstractOperation) = _apply_ops!(f, _qcbops([op], _fh(f).qubits))
# applynoise!(frame, noise, i) (src/pauli_frames.jl:136-174)
applynoise!(f::PauliFrameB200, noise, i::Int) = _apply_ops!(f, _qcbops(NoiseOp(noise, [i])))

# copy(frame) (src/pauli_frames.jl:17): same bits and record on the device;
# the copy draws its own noise stream from then on
function Base.copy(f::PauliFrameB200)
    h = _fh(f)
    g = _frame_b200(h.frames, h.qubits, h.nbits)
    _check(ccall((:qcb_frame_copy, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}), _fh(g).ptr, h.ptr, C_NULL))
    g
end

# measurements(frame) (src/pauli_frames.jl:280): the Bool matrix, on the host
function measurements(f::PauliFrameB200)
    h = _fh(f)
    m = Matrix{Bool}(undef, h.frames, h.nbits)
    _check(ccall((:qcb_frame_download_measurements, libqcb), Cint, (Ptr{Cvoid}, Ptr{Bool}, Ptr{Cvoid}),
                 h.ptr, m, C_NULL))
    m
end

"""measurements(frame)[:, bits] gathered on the device (the syndrome columns
a decoder reads, src/ecc/decoder_pipeline.jl:165-166)."""
function measurement_columns(f::PauliFrameB200, bits::AbstractVector{<:Integer})
    h = _fh(f)
    b = UInt32.(bits)
    m = Matrix{Bool}(undef, h.frames, length(b))
    _check(ccall((:qcb_frame_measurement_columns, libqcb), Cint,
                 (Ptr{Cvoid}, Ptr{UInt32}, Csize_t, Ptr{UInt8}, Ptr{Bool}, Ptr{Cvoid}),
                 h.ptr, b, length(b), C_NULL, m, C_NULL))
    m
end

"""evaluate_guesses (src/ecc/decoder_pipeline.jl:172-190) with
measured_faults = measurements(frame)[:, logical_bits], on the device."""
function evaluate_guesses(f::PauliFrameB200, logical_bits::AbstractVector{<:Integer}, guesses::AbstractMatrix,
                          faults_submatrix::AbstractMatrix)
    h = _fh(f)
    lb = UInt32.(logical_bits)
    g = Matrix{Bool}(guesses .% 2 .== 1)
    F = Matrix{Bool}(faults_submatrix .% 2 .== 1)
    fails = Ref{UInt64}(0)
    _check(ccall((:qcb_evaluate_guesses, libqcb), Cint,
                 (Ptr{Cvoid}, Ptr{UInt32}, Csize_t, Ptr{Bool}, Csize_t, Ptr{Bool}, Ref{UInt64}, Ptr{Cvoid}),
                 h.ptr, lb, length(lb), g, size(g, 2), F, fails, C_NULL))
    fails[] / h.frames
end

# ---------------------------------------------------------------- circuits marked for the device
"""on_b200(circuit): the same op list, marked to run on the B200.  It is an
AbstractVector of the ops, so code written for circuits takes it unchanged;
pftrajectories(on_b200(circuit); trajectories, threads) returns a frame on
the device, and ECC.evaluate_decoder(d, nsamples, on_b200(circuit), ...)
then samples there."""
struct B200Circuit{V<:AbstractVector} <: AbstractVector{Any}
    ops::V
end
Base.size(c::B200Circuit) = size(c.ops)
Base.getindex(c::B200Circuit, i::Int) = c.ops[i]
on_b200(circuit::AbstractVector) = B200Circuit(circuit)

# pftrajectories(circuit; trajectories, threads) (src/pauli_frames.jl:193-227):
# _create_pauliframe's sizes (init = 1), a fresh Philox frame, one launch;
# `threads` is accepted for signature parity (the device has one schedule)
function pftrajectories(c::B200Circuit; trajectories=5000, threads=true)
    qmax = maximum((maximum(affectedqubits(g), init=1) for g in c.ops), init=1)
    bmax = maximum((maximum(affectedbits(g), init=1) for g in c.ops), init=1)
    f = _frame_b200(trajectories, qmax, bmax)
    h = _fh(f)
    prog = _program(_qcbops(c.ops, qmax))
    _check(ccall((:qcb_pftrajectories_fresh, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, UInt64, UInt64, Ptr{Cvoid}),
                 h.ptr, prog.handle, h.seed, 0, C_NULL))
    h.seed += 0x9E3779B97F4A7C15
    f
end

# evaluate_decoder (src/ecc/decoder_pipeline.jl:163-170) with the syndrome
# columns gathered and the guesses checked on the device; the decoder's own
# batchdecode runs on the host as in the reference
function ECC.evaluate_decoder(d::ECC.AbstractSyndromeDecoder, nsamples, c::B200Circuit, syndrome_bits,
                              logical_bits, faults_submatrix)
    frames = pftrajectories(c; trajectories=nsamples, threads=true)
    syndromes = measurement_columns(frames, syndrome_bits)
    guesses = ECC.batchdecode(d, syndromes)
    evaluate_guesses(frames, logical_bits, guesses, faults_submatrix)
end

# ---------------------------------------------------------------- tableau storage
mutable struct TabHandle          # owner of one qcb_tableau (rows x W uint64 + phases)
    ptr::Ptr{Cvoid}
    rows::Int
    nqubits::Int
end
function TabHandle(rows::Integer, nqubits::Integer)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _check(ccall((:qcb_tableau_create, libqcb), Cint, (UInt32, UInt32, Ref{Ptr{Cvoid}}), rows, nqubits, h))
    t = TabHandle(h[], rows, nqubits)
    finalizer(x -> ccall((:qcb_tableau_destroy, libqcb), Cint, (Ptr{Cvoid},), x.ptr), t)
end

"""Tableau rows on the device, seen as the reference's `xzs` (W, rows)."""
struct B200Matrix <: AbstractMatrix{UInt64}
    h::TabHandle
end
Base.size(m::B200Matrix) = (2 * cld(m.h.nqubits, 64), m.h.rows)
Base.getindex(::B200Matrix, ::Int, ::Int) = _noscalar()
"""Tableau phases on the device."""
struct B200Phases <: AbstractVector{UInt8}
    h::TabHandle
end
Base.size(p::B200Phases) = (p.h.rows,)
Base.getindex(::B200Phases, ::Int) = _noscalar()
"""A PauliOperator on the device is a one-row tableau."""
struct B200PauliXZ <: AbstractVector{UInt64}
    h::TabHandle
end
Base.size(v::B200PauliXZ) = (2 * cld(v.h.nqubits, 64),)
Base.getindex(::B200PauliXZ, ::Int) = _noscalar()
struct B200PauliPhase <: AbstractArray{UInt8,0}
    h::TabHandle
end
Base.size(::B200PauliPhase) = ()
Base.getindex(::B200PauliPhase) = _noscalar()

const TableauB200 = Tableau{B200Phases,B200Matrix}
const StabilizerB200 = Stabilizer{TableauB200}
const DestabilizerB200 = Destabilizer{TableauB200}
const MixedStabilizerB200 = MixedStabilizer{TableauB200}
const MixedDestabilizerB200 = MixedDestabilizer{TableauB200}
const StateB200 = Union{StabilizerB200,DestabilizerB200,MixedStabilizerB200,MixedDestabilizerB200}
const PauliOperatorB200 = PauliOperator{B200PauliPhase,B200PauliXZ}

_h(t::TableauB200) = t.xzs.h
_h(s::StateB200) = s.tab.xzs.h
_h(p::PauliOperatorB200) = p.xz.h
_kind(::StabilizerB200) = Cint(0)
_kind(::MixedStabilizerB200) = Cint(1)
_kind(::DestabilizerB200) = Cint(2)
_kind(::MixedDestabilizerB200) = Cint(3)
_rank(s::Union{MixedStabilizerB200,MixedDestabilizerB200}) = Int32(s.rank)
_rank(::StateB200) = Int32(0)

function _upload!(h::TabHandle, phases::AbstractVector, xzs::AbstractMatrix)
    eltype(xzs) == UInt64 || throw(ArgumentError("the B200 path stores UInt64 words (got $(eltype(xzs)))"))
    x = Matrix{UInt64}(xzs)                      # (W, rows): rows contiguous, the reference layout
    _check(ccall((:qcb_tableau_upload, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Ptr{UInt64}, Ptr{Cvoid}),
                 h.ptr, Vector{UInt8}(phases), x, C_NULL))
end

function _download(h::TabHandle)
    ph = Vector{UInt8}(undef, h.rows)
    xzs = Matrix{UInt64}(undef, 2 * cld(h.nqubits, 64), h.rows)
    _check(ccall((:qcb_tableau_download, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Ptr{UInt64}, Ptr{Cvoid}),
                 h.ptr, ph, xzs, C_NULL))
    ph, xzs
end

function to_b200(t::Tableau)
    h = TabHandle(length(t.phases), t.nqubits)
    _upload!(h, t.phases, t.xzs)
    Tableau(B200Phases(h), t.nqubits, B200Matrix(h))
end
to_b200(s::Stabilizer) = Stabilizer(to_b200(s.tab))
to_b200(s::Destabilizer) = Destabilizer(to_b200(s.tab))
to_b200(s::MixedStabilizer) = MixedStabilizer(to_b200(s.tab), s.rank)
to_b200(s::MixedDestabilizer) = MixedDestabilizer(to_b200(s.tab), s.rank)
function to_b200(p::PauliOperator)
    h = TabHandle(1, p.nqubits)
    _upload!(h, [p.phase[]], reshape(Vector{UInt64}(p.xz), :, 1))
    PauliOperator(B200PauliPhase(h), p.nqubits, B200PauliXZ(h))
end

function to_cpu(t::TableauB200)
    ph, xzs = _download(_h(t))
    Tableau(ph, t.nqubits, xzs)
end
to_cpu(s::StabilizerB200) = Stabilizer(to_cpu(s.tab))
to_cpu(s::DestabilizerB200) = Destabilizer(to_cpu(s.tab))
to_cpu(s::MixedStabilizerB200) = MixedStabilizer(to_cpu(s.tab), s.rank)
to_cpu(s::MixedDestabilizerB200) = MixedDestabilizer(to_cpu(s.tab), s.rank)
function to_cpu(p::PauliOperatorB200)
    ph, xzs = _download(_h(p))
    PauliOperator(fill(ph[1]), p.nqubits, vec(xzs))
end

# ---------------------------------------------------------------- mul_left! / mul_right!
# qcb_mul_rows (src/mul_leftright.jl:137-245; the KA extension's device
# methods, ext/QuantumCliffordKAExt/mul_leftright.jl:101-460): target rows of
# a, source rows of b, 1-based; phase_src 1 reads the added phase from a
function _mul_rows!(a::TabHandle, arow, count, b::TabHandle, brow, bstep, right::Bool, phase_src, phases::Bool)
    _check(ccall((:qcb_mul_rows, libqcb), Cint,
                 (Ptr{Cvoid}, UInt32, UInt32, Ptr{Cvoid}, UInt32, UInt32, Cint, Cint, Cint, Ptr{UInt8}, Ptr{Cvoid}),
                 a.ptr, arow, count, b.ptr, brow, bstep, right, phase_src, phases, C_NULL, C_NULL))
end

const TabLikeB200 = Union{TableauB200,StateB200}

for (f, right) in ((:mul_left!, false), (:mul_right!, true))
    @eval begin
        # PauliOperator with PauliOperator
        function $f(u::PauliOperatorB200, v::PauliOperatorB200; phases=Val(true))
            u.nqubits == v.nqubits || throw(DimensionMismatch("The two Pauli operators should have the same length!"))
            _mul_rows!(_h(u), 1, 1, _h(v), 1, 0, $right, 0, _b(phases))
            u
        end
        # PauliOperator with row i of a Tableau / stabilizer state
        function $f(u::PauliOperatorB200, v::TabLikeB200, i::Integer; phases=Val(true))
            _mul_rows!(_h(u), 1, 1, _h(v), i, 0, $right, 0, _b(phases))
            u
        end
        # every row of a Tableau / state with a PauliOperator
        function $f(u::TabLikeB200, v::PauliOperatorB200; phases=Val(true))
            _mul_rows!(_h(u), 1, _h(u).rows, _h(v), 1, 0, $right, 0, _b(phases))
            u
        end
        # rows m and i of one tableau (s.phases[i] added, as the reference)
        function $f(s::TableauB200, m::Integer, i::Integer; phases=Val(true))
            _mul_rows!(_h(s), m, 1, _h(s), i, 0, $right, 0, _b(phases))
            s
        end
        # mul_left!(s, m, t, i): the reference adds s.phases[i] (src/mul_leftright.jl:171-175, 183-187)
        function $f(s::TableauB200, m::Integer, t::TableauB200, i::Integer; phases=Val(true))
            _mul_rows!(_h(s), m, 1, _h(t), i, 0, $right, 1, _b(phases))
            s
        end
    end
end
# mul_left!(state, i, j) (src/mul_leftright.jl:194-219): the Destabilizer
# kinds update destabilizer j by i without phase, then stabilizer i by j
function mul_left!(s::StateB200, i::Integer, j::Integer; phases=Val(true))
    _check(ccall((:qcb_mul_left_state, libqcb), Cint, (Ptr{Cvoid}, Cint, UInt32, UInt32, Cint, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), i, j, _b(phases), C_NULL))
    s
end

function prodphase(l::PauliOperatorB200, r::PauliOperatorB200)
    out = Ref{UInt8}(0)
    _check(ccall((:qcb_prodphase, libqcb), Cint, (Ptr{Cvoid}, UInt32, Ptr{Cvoid}, UInt32, Ref{UInt8}, Ptr{Cvoid}),
                 _h(l).ptr, 1, _h(r).ptr, 1, out, C_NULL))
    out[]
end
function comm(l::PauliOperatorB200, r::PauliOperatorB200)
    out = Ref{UInt8}(0)
    _check(ccall((:qcb_comm, libqcb), Cint, (Ptr{Cvoid}, UInt32, Ptr{Cvoid}, UInt32, Ref{UInt8}, Ptr{Cvoid}),
                 _h(l).ptr, 1, _h(r).ptr, 1, out, C_NULL))
    out[]
end

function rowswap!(s::StateB200, i::Integer, j::Integer; phases=Val(true))
    _check(ccall((:qcb_rowswap, libqcb), Cint, (Ptr{Cvoid}, Cint, UInt32, UInt32, Cint, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), i, j, _b(phases), C_NULL))
    s
end

# ---------------------------------------------------------------- canonical forms
# canonicalize! on the whole state: the Destabilizer kinds carry their
# destabilizer rows through the row swaps and products
function canonicalize!(s::StateB200; phases::Bool=true, ranks::Bool=false)
    rx, rz = Ref{Int32}(0), Ref{Int32}(0)
    _check(ccall((:qcb_canonicalize_state, libqcb), Cint, (Ptr{Cvoid}, Cint, Int32, Cint, Ref{Int32}, Ref{Int32}, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), _rank(s), phases, rx, rz, C_NULL))
    ranks ? (s, Int(rx[]), Int(rz[])) : s
end

function canonicalize_rref!(s::StateB200, colindices; phases::Bool=true)
    cols = UInt32.(collect(colindices))
    i = Ref{Int32}(0)
    _check(ccall((:qcb_canonicalize_rref, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Int32, Ptr{UInt32}, Csize_t, Cint, Ref{Int32}, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), _rank(s), cols, length(cols), phases, i, C_NULL))
    s, Int(i[])
end
canonicalize_rref!(s::StateB200; phases::Bool=true) = canonicalize_rref!(s, 1:nqubits(s); phases)

function canonicalize_gott!(s::StabilizerB200; phases::Bool=true)
    n = nqubits(s)
    r, sz = Ref{Int32}(0), Ref{Int32}(0)
    xperm, zperm = Vector{UInt32}(undef, n), Vector{UInt32}(undef, n)
    _check(ccall((:qcb_canonicalize_gott, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, Ref{Int32}, Ptr{UInt32}, Ptr{UInt32}, Ptr{Cvoid}),
                 _h(s).ptr, phases, r, sz, xperm, zperm, C_NULL))
    s, Int(r[]), Int(sz[]), Int.(xperm), Int.(zperm)
end

function permutesystems!(s::StateB200, perm::AbstractVector)
    p = UInt32.(perm)
    _check(ccall((:qcb_permutesystems, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt32}, Ptr{Cvoid}), _h(s).ptr, p, C_NULL))
    s
end

# generate!(pauli, stabilizer) (src/project_trace_reset.jl:37-81)
function generate!(p::PauliOperatorB200, s::StabilizerB200; phases::Val{B}=Val(true), saveindices::Val{S}=Val(true)) where {B,S}
    ok = Ref{Int32}(0)
    used = Vector{Int32}(undef, nqubits(s))
    nused = Ref{UInt32}(0)
    _check(ccall((:qcb_generate, libqcb), Cint,
                 (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ref{Int32}, Ptr{Int32}, UInt32, Ref{UInt32}, Ptr{Cvoid}),
                 _h(p).ptr, _h(s).ptr, B, ok, used, length(used), nused, C_NULL))
    ok[] == 0 && return nothing
    S ? (p, Int.(used[1:nused[]])) : p
end

# ---------------------------------------------------------------- projections
function project!(s::StateB200, p::PauliOperatorB200; keep_result::Bool=true, phases::Bool=true)
    rank = Ref{Int32}(_rank(s))
    anti, res, done = Ref{Int32}(0), Ref{Int32}(0), Ref{UInt32}(0)
    _check(ccall((:qcb_project, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, Ptr{Cvoid}, Cint, Cint, Ref{Int32}, Ref{Int32}, Ref{UInt32}, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), rank, _h(p).ptr, keep_result, phases, anti, res, done, C_NULL))
    s isa Union{MixedStabilizerB200,MixedDestabilizerB200} && (s.rank = rank[])
    s, Int(anti[]), res[] < 0 ? nothing : UInt8(res[])
end

# projectX! / projectZ! / projectY!: basis 1 / 2 / 3
function _project_qubit!(s::StateB200, basis, qubit::Int; keep_result::Bool=true, phases::Bool=true)
    rank = Ref{Int32}(_rank(s))
    anti, res, done = Ref{Int32}(0), Ref{Int32}(0), Ref{UInt32}(0)
    q = Ref{UInt32}(qubit)
    _check(ccall((:qcb_project_qubit, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, UInt32, Ref{UInt32}, Csize_t, Cint, Cint, Ref{Int32}, Ref{Int32},
                  Ref{UInt32}, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), rank, basis, q, 1, keep_result, phases, anti, res, done, C_NULL))
    s isa Union{MixedStabilizerB200,MixedDestabilizerB200} && (s.rank = rank[])
    s, Int(anti[]), res[] < 0 ? nothing : UInt8(res[])
end
projectX!(s::StateB200, qubit::Int; kw...) = _project_qubit!(s, 1, qubit; kw...)
projectZ!(s::StateB200, qubit::Int; kw...) = _project_qubit!(s, 2, qubit; kw...)
projectY!(s::StateB200, qubit::Int; kw...) = _project_qubit!(s, 3, qubit; kw...)

# projectXrand! and friends: the undetermined sign comes from the task RNG,
# drawn here and handed to the device
function _projectrand!(s::StateB200, basis, qubit::Int)
    rank = Ref{Int32}(_rank(s))
    anti, res, done = Ref{Int32}(0), Ref{Int32}(0), Ref{UInt32}(0)
    q, rp = Ref{UInt32}(qubit), Ref{UInt8}(rand((0x0, 0x2)))
    _check(ccall((:qcb_projectrand, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, Ptr{Cvoid}, UInt32, Ref{UInt32}, Csize_t, Ref{UInt8}, Ref{Int32},
                  Ref{Int32}, Ref{UInt32}, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), rank, C_NULL, basis, q, 1, rp, anti, res, done, C_NULL))
    s isa Union{MixedStabilizerB200,MixedDestabilizerB200} && (s.rank = rank[])
    s, UInt8(res[])
end
projectXrand!(s::StateB200, qubit::Int) = _projectrand!(s, 1, qubit)
projectZrand!(s::StateB200, qubit::Int) = _projectrand!(s, 2, qubit)
projectYrand!(s::StateB200, qubit::Int) = _projectrand!(s, 3, qubit)

# expect(p, s) (src/project_trace_reset.jl:743-751) on a device state, which
# is not modified
function expect(p::PauliOperatorB200, s::StateB200)
    out = Ref{Int32}(0)
    _check(ccall((:qcb_expect, libqcb), Cint, (Ptr{Cvoid}, Cint, Int32, Ptr{Cvoid}, Ref{Int32}, Ptr{Cvoid}),
                 _h(s).ptr, _kind(s), _rank(s), _h(p).ptr, out, C_NULL))
    out[] < 0 ? 0 : (1, im, -1, -im)[out[] + 1]
end

# ---------------------------------------------------------------- apply!
function apply!(s::Union{StateB200,TableauB200}, gate::AbstractSymbolicOperator; phases::Bool=true)
    ops = _qcbops(gate)
    _check(ccall((:qcb_apply_gates, libqcb), Cint, (Ptr{Cvoid}, Ptr{QcbOp}, Csize_t, Cint, Ptr{Cvoid}),
                 _h(s).ptr, ops, length(ops), phases, C_NULL))
    s
end

function apply!(s::Union{StateB200,TableauB200}, c::CliffordOperator; phases::Bool=true)
    ct = to_b200(c.tab)
    _check(ccall((:qcb_apply_dense, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}),
                 _h(s).ptr, _h(ct).ptr, phases, C_NULL))
    s
end

function __init__()
    _check(ccall((:qcb_init, libqcb), Cint, (Cint,), 0))
end

end # module
