# QuantumCliffordB200Ext -- Julia package extension that routes QuantumClifford's
# bit-packed tableau / Pauli-frame hot path to libqcb200 (B200, sm_100a) through
# `ccall`.  It plays the role ext/QuantumCliffordGPUExt plays for CUDA.jl arrays:
# methods are selected by dispatch on the device-backed storage types defined here.
#
# Not exercised in this repository (no Julia toolchain here); the same C ABI is
# exercised by the Python mirror in ../qcb200 and its tests.
module QuantumCliffordB200Ext

using QuantumClifford
import QuantumClifford: apply!, pftrajectories, mul_left!, canonicalize!, project!,
    canonicalize_rref!, canonicalize_gott!, permutesystems!, projectX!, projectY!, projectZ!,
    projectXrand!, projectYrand!, projectZrand!,
    measurements, PauliFrame, Stabilizer, MixedDestabilizer, Destabilizer, MixedStabilizer,
    PauliOperator, Tableau, nqubits, tab, CliffordOperator, AbstractOperation,
    SingleQubitOperator, ClassicalXOR, PauliMeasurement

const libqcb = get(ENV, "QCB200_LIB", joinpath(@__DIR__, "..", "lib", "libqcb200.so"))

# ---------------------------------------------------------------- errors
const QCB_OK = Cint(0)

function _check(st::Cint)
    st == QCB_OK && return nothing
    buf = Vector{UInt8}(undef, 4096)
    ccall((:qcb_last_error, libqcb), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
    msg = unsafe_string(pointer(buf))
    st == 1 && throw(DimensionMismatch(msg))
    st == 2 && throw(BoundsError(msg))
    (st == 3 || st == 4) && throw(ArgumentError(msg))
    st == 9 && throw(QuantumClifford.BadDataStructure(msg, :project!, :Destabilizer))
    error("libqcb200 status $st: $msg")
end

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
_qcbops(op::NoisyGate) = vcat(_qcbops(op.gate), _qcbops(NoiseOp(op.noise, collect(QuantumClifford.affectedqubits(op.gate)))))
# NoiseOpAll (src/noise.jl:173-176, 192-195): the noise on qubits 1..n of the
# frame (n = nqubits(frame), the hidden ancilla excluded)
_qcbops(op::NoiseOpAll, n::Integer) = _qcbops(NoiseOp(op.noise, collect(1:n)))
_qcbops(op, n::Integer) = _qcbops(op)
_qcbops(circuit::AbstractVector, n::Integer=0) = reduce(vcat, (_qcbops(op, n) for op in circuit); init=QcbOp[])

# ---------------------------------------------------------------- programs
mutable struct B200Program
    handle::Ptr{Cvoid}
    function B200Program(circuit, n::Integer=0)
        ops = _qcbops(circuit, n)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        _check(ccall((:qcb_program_compile, libqcb), Cint, (Ptr{QcbOp}, Csize_t, Ref{Ptr{Cvoid}}), ops, length(ops), h))
        p = new(h[])
        finalizer(x -> ccall((:qcb_program_destroy, libqcb), Cint, (Ptr{Cvoid},), x.handle), p)
    end
end

const _programs = IdDict{Any,B200Program}()   # circuits compiled once
_program(circuit, n::Integer=0) = get!(() -> B200Program(circuit, n), _programs, (circuit, n))

# ---------------------------------------------------------------- frames
"""Device Pauli frame; `to_b200(PauliFrame(...))` or `B200Frame(frames, qubits, bits)`."""
mutable struct B200Frame
    handle::Ptr{Cvoid}
    frames::Int
    qubits::Int
    nbits::Int
    seed::UInt64
end

function B200Frame(frames::Integer, qubits::Integer, bits::Integer; seed::Integer=rand(UInt64))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _check(ccall((:qcb_frame_create, libqcb), Cint, (UInt64, UInt32, UInt32, Ref{Ptr{Cvoid}}), frames, qubits, bits, h))
    f = B200Frame(h[], frames, qubits, bits, UInt64(seed))
    finalizer(x -> ccall((:qcb_frame_destroy, libqcb), Cint, (Ptr{Cvoid},), x.handle), f)
    _check(ccall((:qcb_frame_init_z, libqcb), Cint, (Ptr{Cvoid}, UInt64, UInt64, Ptr{Cvoid}), f.handle, f.seed, 0, C_NULL))
    f
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

function pftrajectories(f::B200Frame, circuit)
    src = Ref(NoiseSource(0, 0, f.seed, 0, C_NULL, 0, C_NULL))
    _check(ccall((:qcb_pftrajectories, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{NoiseSource}, Ptr{Cvoid}),
                 f.handle, _program(circuit, f.qubits).handle, src, C_NULL))
    f.seed += 0x9E3779B97F4A7C15   # next call draws fresh randomness
    f
end

apply!(f::B200Frame, op::AbstractOperation) = pftrajectories(f, [op])

# copy(frame) (src/pauli_frames.jl:17): same bits and record on the device;
# the copy draws its own noise stream from then on
function Base.copy(f::B200Frame)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _check(ccall((:qcb_frame_create, libqcb), Cint, (UInt64, UInt32, UInt32, Ref{Ptr{Cvoid}}), f.frames, f.qubits, f.nbits, h))
    g = B200Frame(h[], f.frames, f.qubits, f.nbits, rand(UInt64))
    finalizer(x -> ccall((:qcb_frame_destroy, libqcb), Cint, (Ptr{Cvoid},), x.handle), g)
    _check(ccall((:qcb_frame_copy, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}), g.handle, f.handle, C_NULL))
    g
end

function measurements(f::B200Frame)
    m = Matrix{Bool}(undef, f.frames, f.nbits)
    _check(ccall((:qcb_frame_download_measurements, libqcb), Cint, (Ptr{Cvoid}, Ptr{Bool}, Ptr{Cvoid}),
                 f.handle, m, C_NULL))
    m
end

# The decoder hand-off (src/ecc/decoder_pipeline.jl:163-190): the syndrome
# columns for batchdecode, and evaluate_guesses on the device
function measurements(f::B200Frame, bits::AbstractVector{<:Integer})
    b = UInt32.(bits)
    m = Matrix{Bool}(undef, f.frames, length(b))
    _check(ccall((:qcb_frame_measurement_columns, libqcb), Cint,
                 (Ptr{Cvoid}, Ptr{UInt32}, Csize_t, Ptr{UInt8}, Ptr{Bool}, Ptr{Cvoid}),
                 f.handle, b, length(b), C_NULL, m, C_NULL))
    m
end

function evaluate_guesses(f::B200Frame, logical_bits::AbstractVector{<:Integer}, guesses::AbstractMatrix{Bool},
                          faults_submatrix::AbstractMatrix)
    lb = UInt32.(logical_bits)
    g = Matrix{Bool}(guesses)
    F = Matrix{Bool}(faults_submatrix .% 2 .== 1)
    fails = Ref{UInt64}(0)
    _check(ccall((:qcb_evaluate_guesses, libqcb), Cint,
                 (Ptr{Cvoid}, Ptr{UInt32}, Csize_t, Ptr{Bool}, Csize_t, Ptr{Bool}, Ref{UInt64}, Ptr{Cvoid}),
                 f.handle, lb, length(lb), g, size(g, 2), F, fails, C_NULL))
    fails[] / f.frames
end

"""The frame tableau back in the reference fastcolumn layout (UInt64)."""
function QuantumClifford.PauliFrame(f::B200Frame)
    W = 2 * cld(f.qubits + 1, 64)
    xzs = Matrix{UInt64}(undef, f.frames, W)          # frames contiguous per word
    _check(ccall((:qcb_frame_download_xzs, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Ptr{Cvoid}), f.handle, xzs, C_NULL))
    stab = Stabilizer(Tableau(zeros(UInt8, f.frames), f.qubits + 1, collect(xzs')))
    PauliFrame(fastcolumn(stab), measurements(f))
end

to_b200(f::PauliFrame; seed::Integer=rand(UInt64)) = begin
    g = B200Frame(length(f), nqubits(f), size(f.measurements, 2); seed)
    xzs = collect(permutedims(tab(f.frame).xzs))     # frames x W, frames contiguous per word
    _check(ccall((:qcb_frame_upload_xzs, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt64}, Ptr{Cvoid}), g.handle, xzs, C_NULL))
    g
end

"""pftrajectories(circuit; trajectories) on the device in one call."""
function pftrajectories_b200(circuit; trajectories=5000, seed::Integer=rand(UInt64))
    qmax = maximum((maximum(affectedqubits(g), init=1) for g in circuit))
    bmax = maximum((maximum(affectedbits(g), init=1) for g in circuit))
    f = B200Frame(trajectories, qmax, bmax; seed)
    pftrajectories(f, circuit)
end

# ---------------------------------------------------------------- tableaux
mutable struct B200Tableau
    handle::Ptr{Cvoid}
    rows::Int
    nqubits::Int
end

function B200Tableau(t::Tableau)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _check(ccall((:qcb_tableau_create, libqcb), Cint, (UInt32, UInt32, Ref{Ptr{Cvoid}}), length(t), t.nqubits, h))
    d = B200Tableau(h[], length(t), t.nqubits)
    finalizer(x -> ccall((:qcb_tableau_destroy, libqcb), Cint, (Ptr{Cvoid},), x.handle), d)
    xzs = convert(Matrix{UInt64}, t.xzs)          # (W, rows) column-major: rows contiguous
    _check(ccall((:qcb_tableau_upload, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Ptr{UInt64}, Ptr{Cvoid}),
                 d.handle, convert(Vector{UInt8}, t.phases), xzs, C_NULL))
    d
end
B200Tableau(p::PauliOperator) = B200Tableau(Tableau([p]))

function download!(t::Tableau, d::B200Tableau)
    ph = Vector{UInt8}(undef, d.rows)
    xzs = Matrix{UInt64}(undef, size(t.xzs)...)
    _check(ccall((:qcb_tableau_download, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Ptr{UInt64}, Ptr{Cvoid}),
                 d.handle, ph, xzs, C_NULL))
    t.phases .= ph
    t.xzs .= xzs
    t
end

"""A state whose tableau lives on the B200: `to_b200(s)`, `to_cpu(s)`."""
struct B200State{S}
    host::S             # host object (shape, kind, rank)
    dev::B200Tableau
end
to_b200(s::Union{Stabilizer,Destabilizer,MixedStabilizer,MixedDestabilizer}) = B200State(copy(s), B200Tableau(tab(s)))
to_b200(p::PauliOperator) = B200State(copy(p), B200Tableau(p))
to_cpu(s::B200State) = (download!(tab(s.host), s.dev); s.host)

_kind(::Stabilizer) = 0
_kind(::MixedStabilizer) = 1
_kind(::Destabilizer) = 2
_kind(::MixedDestabilizer) = 3

function mul_left!(r::B200State{<:PauliOperator}, l::B200State{<:PauliOperator}; phases::Val{B}=Val(true)) where B
    ph = Ref{UInt8}(0)
    _check(ccall((:qcb_mul_left_pauli, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ref{UInt8}, Ptr{Cvoid}),
                 r.dev.handle, l.dev.handle, B, ph, C_NULL))
    B && (r.host.phase[] = ph[])
    r
end

_rank(h) = h isa Union{MixedStabilizer,MixedDestabilizer} ? Int32(h.rank) : Int32(0)

# canonicalize! on the whole state: the Destabilizer kinds carry their
# destabilizer rows through the row swaps and products
function canonicalize!(s::B200State; phases::Bool=true, ranks::Bool=false)
    h = s.host
    rx, rz = Ref{Int32}(0), Ref{Int32}(0)
    _check(ccall((:qcb_canonicalize_state, libqcb), Cint, (Ptr{Cvoid}, Cint, Int32, Cint, Ref{Int32}, Ref{Int32}, Ptr{Cvoid}),
                 s.dev.handle, _kind(h), _rank(h), phases, rx, rz, C_NULL))
    ranks ? (s, Int(rx[]), Int(rz[])) : s
end

function canonicalize_rref!(s::B200State, colindices; phases::Bool=true)
    h = s.host
    cols = UInt32.(collect(colindices))
    i = Ref{Int32}(0)
    _check(ccall((:qcb_canonicalize_rref, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Int32, Ptr{UInt32}, Csize_t, Cint, Ref{Int32}, Ptr{Cvoid}),
                 s.dev.handle, _kind(h), _rank(h), cols, length(cols), phases, i, C_NULL))
    s, Int(i[])
end
canonicalize_rref!(s::B200State; phases::Bool=true) = canonicalize_rref!(s, 1:nqubits(s.host); phases)

function canonicalize_gott!(s::B200State{<:Stabilizer}; phases::Bool=true)
    n = nqubits(s.host)
    r, sz = Ref{Int32}(0), Ref{Int32}(0)
    xperm, zperm = Vector{UInt32}(undef, n), Vector{UInt32}(undef, n)
    _check(ccall((:qcb_canonicalize_gott, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, Ref{Int32}, Ptr{UInt32}, Ptr{UInt32}, Ptr{Cvoid}),
                 s.dev.handle, phases, r, sz, xperm, zperm, C_NULL))
    s, Int(r[]), Int(sz[]), Int.(xperm), Int.(zperm)
end

function permutesystems!(s::B200State, perm::AbstractVector)
    p = UInt32.(perm)
    _check(ccall((:qcb_permutesystems, libqcb), Cint, (Ptr{Cvoid}, Ptr{UInt32}, Ptr{Cvoid}), s.dev.handle, p, C_NULL))
    s
end

# projectX! / projectZ! / projectY!: basis 1 / 2 / 3
function _project_qubit!(s::B200State, basis, qubit::Int; keep_result::Bool=true, phases::Bool=true)
    h = s.host
    rank = Ref{Int32}(_rank(h))
    anti, res, done = Ref{Int32}(0), Ref{Int32}(0), Ref{UInt32}(0)
    q = Ref{UInt32}(qubit)
    _check(ccall((:qcb_project_qubit, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, UInt32, Ref{UInt32}, Csize_t, Cint, Cint, Ref{Int32}, Ref{Int32},
                  Ref{UInt32}, Ptr{Cvoid}),
                 s.dev.handle, _kind(h), rank, basis, q, 1, keep_result, phases, anti, res, done, C_NULL))
    h isa Union{MixedStabilizer,MixedDestabilizer} && (h.rank = rank[])
    s, Int(anti[]), res[] < 0 ? nothing : UInt8(res[])
end
projectX!(s::B200State, qubit::Int; kw...) = _project_qubit!(s, 1, qubit; kw...)
projectZ!(s::B200State, qubit::Int; kw...) = _project_qubit!(s, 2, qubit; kw...)
projectY!(s::B200State, qubit::Int; kw...) = _project_qubit!(s, 3, qubit; kw...)

# projectXrand! and friends: the undetermined sign comes from the task RNG,
# drawn here and handed to the device
function _projectrand!(s::B200State, basis, qubit::Int)
    h = s.host
    rank = Ref{Int32}(_rank(h))
    anti, res, done = Ref{Int32}(0), Ref{Int32}(0), Ref{UInt32}(0)
    q, rp = Ref{UInt32}(qubit), Ref{UInt8}(rand((0x0, 0x2)))
    _check(ccall((:qcb_projectrand, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, Ptr{Cvoid}, UInt32, Ref{UInt32}, Csize_t, Ref{UInt8}, Ref{Int32},
                  Ref{Int32}, Ref{UInt32}, Ptr{Cvoid}),
                 s.dev.handle, _kind(h), rank, C_NULL, basis, q, 1, rp, anti, res, done, C_NULL))
    h isa Union{MixedStabilizer,MixedDestabilizer} && (h.rank = rank[])
    s, UInt8(res[])
end
projectXrand!(s::B200State, qubit::Int) = _projectrand!(s, 1, qubit)
projectZrand!(s::B200State, qubit::Int) = _projectrand!(s, 2, qubit)
projectYrand!(s::B200State, qubit::Int) = _projectrand!(s, 3, qubit)

function project!(s::B200State, p::B200State{<:PauliOperator}; keep_result::Bool=true, phases::Bool=true)
    h = s.host
    rank = Ref{Int32}(h isa Union{MixedStabilizer,MixedDestabilizer} ? h.rank : 0)
    anti, res, done = Ref{Int32}(0), Ref{Int32}(0), Ref{UInt32}(0)
    _check(ccall((:qcb_project, libqcb), Cint,
                 (Ptr{Cvoid}, Cint, Ref{Int32}, Ptr{Cvoid}, Cint, Cint, Ref{Int32}, Ref{Int32}, Ref{UInt32}, Ptr{Cvoid}),
                 s.dev.handle, _kind(h), rank, p.dev.handle, keep_result, phases, anti, res, done, C_NULL))
    h isa Union{MixedStabilizer,MixedDestabilizer} && (h.rank = rank[])
    s, Int(anti[]), res[] < 0 ? nothing : UInt8(res[])
end

# expect(p, s) (src/project_trace_reset.jl:743-751) on a device state, which
# is not modified
function QuantumClifford.expect(p::B200State{<:PauliOperator}, s::B200State)
    h = s.host
    out = Ref{Int32}(0)
    _check(ccall((:qcb_expect, libqcb), Cint, (Ptr{Cvoid}, Cint, Int32, Ptr{Cvoid}, Ref{Int32}, Ptr{Cvoid}),
                 s.dev.handle, _kind(h), _rank(h), p.dev.handle, out, C_NULL))
    out[] < 0 ? 0 : (1, im, -1, -im)[out[] + 1]
end

function apply!(s::B200State, gate::AbstractSymbolicOperator; phases::Bool=true)
    ops = _qcbops(gate)
    _check(ccall((:qcb_apply_gates, libqcb), Cint, (Ptr{Cvoid}, Ptr{QcbOp}, Csize_t, Cint, Ptr{Cvoid}),
                 s.dev.handle, ops, length(ops), phases, C_NULL))
    s
end

function apply!(s::B200State, c::CliffordOperator; phases::Bool=true)
    cd = B200Tableau(tab(c))
    _check(ccall((:qcb_apply_dense, libqcb), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}),
                 s.dev.handle, cd.handle, phases, C_NULL))
    s
end

function __init__()
    _check(ccall((:qcb_init, libqcb), Cint, (Cint,), 0))
end

end # module
