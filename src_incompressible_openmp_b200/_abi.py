"""ctypes mirrors of the POD structs and enums declared in include/mpcd_c.h.

Field order and types must match the C header exactly; tests check sizeof() of each struct
against the library's own view (mpcd_abi_sizes).
"""
import ctypes as C

MPCD_OK = 0
STATUS_NAMES = {
    0: "MPCD_OK", 1: "MPCD_ERR_INVALID_ARG", 2: "MPCD_ERR_CUDA", 3: "MPCD_ERR_UNSUPPORTED_BC",
    4: "MPCD_ERR_DEVICE", 5: "MPCD_ERR_NO_DEVICE", 6: "MPCD_ERR_CAPACITY", 7: "MPCD_ERR_STATE",
}

BC_MODES = {"periodic": 0, "thermalize": 1, "bounceback": 2, "specular": 3}
BC_UNKNOWN = -1
THR_MODES = {"coef": 0, "1+coef": 1}
LAYOUT_MODES = {"base": 0, "shifted": 1, "single_full": 2}

_I = C.c_int32
_D = C.c_double


class ParamsC(C.Structure):
    _fields_ = [
        ("Nx", _I), ("Ny", _I), ("Nc", _I), ("n", _I),
        ("Lx", _D), ("Ly", _D), ("dt", _D), ("a0", _D),
        ("alpha", _D), ("kBT", _D), ("g", _D), ("bodyForceX", _D),
        ("useThermostat", _I), ("keepMeanFlow", _I),
        ("boundary_left", _I), ("boundary_right", _I), ("boundary_bottom", _I), ("boundary_top", _I),
        ("Utop", _D), ("Ubottom", _D), ("wallSigma", _D),
        ("noSurfaceCase", _I), ("redistributionEnableSurfaceTopology", _I), ("redistributionWallWettingEnabled", _I),
        ("useInterfaceVelocityReorientation", _I), ("useIncompressibleRedistribution", _I),
        ("redistribAfterCollision", _I), ("useZoneRedistribution", _I),
        ("zoneTileNx", _I), ("zoneTileNy", _I),
        ("zoneUseShiftedSecondPass", _I), ("zonePassthroughMode", _I), ("zoneSingleFullDomainMode", _I),
        ("enableMomentumCorrectionPostRedistribution", _I),
        ("gamma", _D), ("coef", _D),
        ("highMode", _I), ("lowMode", _I),
        ("maxRedistribPasses", _I), ("useLocalFluidFractionThresholds", _I),
        ("fluidFracGain", _D), ("lowThrFloor", _D), ("highThrFloor", _D), ("lowThrBulkOverride", _D),
        ("useLiquidClosure", _I), ("useOptimalBetaRepair", _I),
        ("betaRepair", _D), ("betaEOS", _D), ("Kvirial", _D),
        ("smoothPdriveAtInterzone", _I), ("smoothPdriveInterzoneWidthCells", _I),
        ("smoothPdriveInterzoneBlend", _D),
        ("smoothPdriveIncludeShiftedLayouts", _I), ("reserved0", _I),
    ]


class WallInfoC(C.Structure):
    _fields_ = [("nBot", _I), ("nTop", _I), ("nLeft", _I), ("nRight", _I)] + [
        (k, _D) for k in ("dEwall", "dPxBot", "dPxTop", "dPyBot", "dPyTop", "dPxLeft", "dPxRight", "dPyLeft", "dPyRight")
    ]


class PassMetricsC(C.Structure):
    _fields_ = [
        ("nZones", _I), ("nThreadsRequested", _I), ("nThreadsUsed", _I),
        ("nParticlesMovedDense", _I), ("nParticlesMovedSparse", _I), ("reserved0", _I),
        ("corrRmsDU", _D), ("corrMaxDU", _D),
    ] + [(k, _D) for k in ("timeLayout", "timeZoneExtract", "timeSnapshot", "timeAlloc", "timeKernel", "timePack", "timeMerge")]


CLOSURE_DOUBLE_FIELDS = (
    "betaRepairOpt", "betaRepairApplied", "betaRepairNum", "betaRepairDen", "betaEOSApplied",
    "meanPdriveRaw", "meanPdrive", "rmsRepairDU", "meanAbsRepairDU", "maxRepairDU",
    "rmsEOSDU", "maxEOSDU", "momentumDeltaX", "momentumDeltaY",
)


class ClosureMetricsC(C.Structure):
    _fields_ = [(k, _D) for k in CLOSURE_DOUBLE_FIELDS] + [("nMaskedInterzoneCells", _I), ("reserved0", _I)]


FIELD_NAMES = ("Ux", "Uy", "Px", "Py", "T", "rho", "Pkin", "Pvir", "P", "rhoTarget")
_DP = C.POINTER(C.c_double)


class CellFieldsC(C.Structure):
    _fields_ = [("N", C.POINTER(C.c_int32))] + [(k, _DP) for k in FIELD_NAMES]


class ClosureDetailC(C.Structure):
    _fields_ = [
        ("repairedX", _DP), ("repairedV", _DP),
        ("refFields", CellFieldsC), ("redFields", CellFieldsC), ("repairedFields", CellFieldsC), ("outFields", CellFieldsC),
        ("pdriveRaw", _DP), ("pdrive", _DP), ("duRepairX", _DP), ("duRepairY", _DP), ("duEOSX", _DP), ("duEOSY", _DP),
        ("interzoneMask", C.POINTER(C.c_int32)),
    ]


STEP_DOUBLE_FIELDS = (
    "occStd", "outBand", "meanKinetic", "meanUx", "meanUy", "Qx",
    "baseOccStd", "baseOutBand", "shiftedOccStd", "shiftedOutBand",
    "meanVelocityX", "meanVelocityY",
    "timeStepTotal", "timeRefBuild", "timeBase", "timeShifted", "timeClosure", "timeDiagnostics",
)


class StepMetricsC(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("wall", WallInfoC), ("base", PassMetricsC), ("shifted", PassMetricsC),
        ("closure", ClosureMetricsC),
    ] + [(k, _D) for k in STEP_DOUBLE_FIELDS]


def struct_to_dict(s):
    out = {}
    for name, _ in s._fields_:
        val = getattr(s, name)
        if isinstance(val, C.Structure):
            val = struct_to_dict(val)
        out[name] = val
    return out


ABI_STRUCTS = {
    "mpcd_params_c": ParamsC, "mpcd_wallinfo_c": WallInfoC, "mpcd_pass_metrics_c": PassMetricsC,
    "mpcd_closure_metrics_c": ClosureMetricsC, "mpcd_cellfields_c": CellFieldsC,
    "mpcd_closure_detail_c": ClosureDetailC, "mpcd_step_metrics_c": StepMetricsC,
}
