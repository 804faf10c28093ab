"""qcb200 -- host-side mirror of QuantumClifford.jl's bit-packed tableau /
Pauli-frame API over libqcb200 (the B200 C ABI in include/qcb200.h).

Julia names map to Python ones with ``!`` spelled as a trailing underscore:
``mul_left!`` -> ``mul_left_``, ``canonicalize!`` -> ``canonicalize_``,
``project!`` -> ``project_``, ``apply!`` -> ``apply_``, ``pauliframe!`` ->
``pauliframe_``.
"""
from ._lib import (  # noqa: F401
    QCBError, DimensionMismatch, BoundsError, ArgumentError, BadDataStructure, lib, check, ensure_init,
    exported_symbols, LIB_PATH, OP_DTYPE, EVENT_DTYPE,
)
from .ops import (  # noqa: F401
    Op, OP, sId1, sHadamard, sPhase, sInvPhase, sX, sY, sZ, sSQRTX, sInvSQRTX, sSQRTY, sInvSQRTY,
    sHadamardXY, sHadamardYZ, sCXYZ, sCZYX, SingleQubitOperator, sCNOT, sCPHASE, sSWAP, sZCX, sZCY, sZCZ, sXCX, sXCY, sXCZ,
    sYCX, sYCY, sYCZ, sSWAPCX, sInvSWAPCX, sISWAP, sInvISWAP, sCZSWAP, sCXSWAP, sZCrY, sInvZCrY, sSQRTZZ,
    sInvSQRTZZ, sSQRTXX, sInvSQRTXX, sSQRTYY, sInvSQRTYY, sMZ, sMRZ, sMX, sMRX, ClassicalXOR, PauliMeasurement, PauliError, NoiseOp, PauliNoise, UnbiasedUncorrelatedNoise,
    DepolarizationNoise, NoisyGate, NoiseOpAll, to_array, count_updates, affected_counts,
)
from .frames import (  # noqa: F401
    PauliFrame, Program, Masks, sample_masks, pftrajectories, pauliframe_, measurements,
    pftrajectories_record, unpack_record, pack_record, evaluate_guesses, Batch, tune_tile, tune_walker,
    tune_walker_clear, Server,
)
from .tableau import (  # noqa: F401
    Tableau, PauliOperator, Stabilizer, MixedStabilizer, Destabilizer, MixedDestabilizer, CliffordOperator,
    P, S, T, tCNOT, tensor_pow, one_destabilizer, one_mixed_destabilizer, random_clifford_ops,
    mul_left_, mul_right_, mul_left_row_, prodphase, comm, canonicalize_, project_, generate_, apply_, DeviceTableau,
    canonicalize_rref_, canonicalize_gott_, permutesystems_, projectX_, projectY_, projectZ_,
    projectrand_, projectXrand_, projectYrand_, projectZrand_, CanonBatch, expect, rowswap_,
)
from . import circuits  # noqa: F401
from .randoms import random_destabilizer, random_stabilizer, random_clifford, random_paulis  # noqa: F401
