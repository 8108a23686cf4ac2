"""The emsart.cfg configuration surface (src/EmSART/utils/Config.cpp).

`parse_config` reads `name = value` lines as the reference's parser does
(lines starting with '#' are comments; `name = (` opens a group that a line
with ')' closes; values are trimmed) and `EmSartConfig.from_file` turns the
symbols into the settings the reconstruction path reads, with the
reference's defaults and value syntax: booleans are yes/true (any case of
Yes/YES/True/TRUE), vectors may be wrapped in (), [] or {} and separated by
spaces, commas or semicolons, VoxelSize is one value or three,
WBPFilter/ProjectionNormalization take the reference's names.
"""
from __future__ import annotations

from dataclasses import dataclass, field


def parse_config(text: str) -> dict:
    """Symbols of a config file (groups flattened, the last value of a name
    wins, as the reference's map does)."""
    symbols = {}
    for raw in text.splitlines():
        line = raw.rstrip("\r\n")
        if len(line) > 2 and not line.startswith("#") and ")" not in line:
            if "=" not in line:
                continue
            name, value = line.split("=", 1)
            name, value = name.strip(), value.strip()
            if value == "(":
                continue
            symbols[name] = value
    return symbols


def _bool(v: str) -> bool:
    return v in ("yes", "Yes", "YES", "true", "True", "TRUE")


def _floats(v: str, strip_dots: bool = False) -> list:
    chars = "([{;)]},"
    if strip_dots:
        chars += "."
    for c in chars:
        v = v.replace(c, " ")
    return [float(x) for x in v.split()]


WBP_FILTERS = {"ramp": 0, "exact": 1, "contrast2": 2, "contrast10": 3, "contrast30": 4}


@dataclass
class EmSartConfig:
    ProjectionFile: str = ""
    OutVolumeFile: str = ""
    MarkerFile: str = ""
    CtfFile: str = ""
    CudaDeviceID: list = field(default_factory=lambda: [0])
    Lambda: float = 1.0
    Iterations: int = 1
    RecDimensions: tuple = (0, 0, 0)
    UseFixPsiAngle: bool = False
    PsiAngle: float = 0.0
    PhiAngle: float = 0.0
    VolumeShift: tuple = (0.0, 0.0, 0.0)
    ReferenceMarker: int = 0
    OverSampling: int = 1
    VoxelSize: tuple = (1.0, 1.0, 1.0)
    AddTiltAngle: float = 0.0
    AddTiltXAngle: float = 0.0
    DimLength: tuple = (0.0, 0.0)
    CutLength: tuple = (0.0, 0.0)
    Crop: tuple = (0.0, 0.0, 0.0, 0.0)
    CropDim: tuple = (0.0, 0.0, 0.0, 0.0)
    SkipFilter: bool = False
    fourFilterLP: int = 800
    fourFilterLPS: int = 200
    fourFilterHP: int = 0
    fourFilterHPS: int = 0
    SIRTCount: int = 1
    CTFBetaFac: tuple = (200.0, 0.0, 0.008, 0.0)
    FP16Volume: bool = False
    WriteVolumeAsFP16: bool = False
    ProjectionScaleFactor: float = 1.0
    WBP: bool = False
    DoseWeighting: bool = False
    AccumulatedDose: list = field(default_factory=list)
    DownWeightTiltsForWBP: bool = False
    SwitchCTFDirectionForIMOD: bool = False
    PhaseFlipOnly: bool = False
    WienerFilterNoiseLevel: float = 0.1
    WBPFilter: int = 0
    CtfMode: bool = False
    Cs: float = 2.7
    Voltage: float = 300.0
    BadPixelValue: float = 10.0
    CorrectBadPixels: bool = True
    ProjectionNormalization: int = 0  # PNM_MEAN
    MagAnisotropy: tuple = (1.0, 0.0)
    IgnoreZShiftForCTF: bool = False
    CTFSliceThickness: float = 50.0
    # EmSARTSubVolumes (SUBVOLREC_MODE keys of utils/Config.cpp:479-494)
    SizeSubVol: int = 0
    VoxelSizeSubVol: float = 0.0
    MotiveList: str = ""
    SubVolPath: str = ""
    ShiftInputFile: str = ""
    BatchSize: int = 0
    MaxShift: int = 0
    NamingConvention: int = 0  # NC_ParticleOnly, 1 NC_TomogramParticle
    ScaleMotivelistShift: float = 1.0
    ScaleMotivelistPosition: float = 1.0
    # EmSartRefine (REFINE_MODE keys of utils/Config.cpp:408-470)
    Reference: str = ""
    ShiftOutputFile: str = ""
    GroupMode: str = "ByGroup"
    GroupSize: int = 0
    MaxDistance: float = 0.0
    SpeedUpDistance: int = 0
    MultiPeakDetection: bool = False
    CCMapFileName: str = ""
    SupportingReferences: list = field(default_factory=list)
    SupportingMotiveLists: list = field(default_factory=list)
    MaxDistanceSupport: float = 0.0

    @classmethod
    def from_text(cls, text: str, subvolumes: bool = False, refine: bool = False) -> "EmSartConfig":
        s = parse_config(text)
        c = cls()

        def req(name):
            if name not in s:
                raise KeyError(f"missing property '{name}'")
            return s[name]

        def opt(name, default=None):
            return s.get(name, default)

        c.ProjectionFile = req("ProjectionFile")
        c.OutVolumeFile = req("OutVolumeFile")
        c.MarkerFile = req("MarkerFile")
        if "CudaDeviceID" in s:
            c.CudaDeviceID = [int(x) for x in _floats(s["CudaDeviceID"])]
        c.Lambda = float(req("Lambda"))
        c.Iterations = int(float(req("Iterations")))
        c.RecDimensions = tuple(int(x) for x in _floats(req("RecDimesions"), strip_dots=True)[:3])
        c.UseFixPsiAngle = _bool(req("UseFixPsiAngle"))
        if c.UseFixPsiAngle:
            c.PsiAngle = float(req("PsiAngle"))
        c.VolumeShift = tuple(_floats(req("VolumeShift"))[:3])
        c.ReferenceMarker = int(float(req("ReferenceMarker")))
        c.OverSampling = int(float(req("OverSampling")))
        c.PhiAngle = float(req("PhiAngle"))
        vs = _floats(req("VoxelSize"))
        c.VoxelSize = tuple(vs[:3]) if len(vs) >= 3 else (vs[0],) * 3
        c.AddTiltAngle = float(opt("AddTiltAngle", "0"))
        c.AddTiltXAngle = float(opt("AddTiltXAngle", "0"))
        c.DimLength = tuple(_floats(req("DimLength"))[:2])
        c.CutLength = tuple(_floats(req("CutLength"))[:2])
        if "Crop" in s:
            c.Crop = tuple(_floats(s["Crop"])[:4])
        if "CropDim" in s:
            c.CropDim = tuple(_floats(s["CropDim"])[:4])
        c.SkipFilter = _bool(req("SkipFilter"))
        c.fourFilterLP = int(float(req("fourFilterLP")))
        c.fourFilterLPS = int(float(req("fourFilterLPS")))
        c.fourFilterHP = int(float(req("fourFilterHP")))
        c.fourFilterHPS = int(float(req("fourFilterHPS")))
        c.SIRTCount = int(float(req("SIRTCount")))
        if "CTFBetaFac" in s and _floats(s["CTFBetaFac"]):
            c.CTFBetaFac = tuple(_floats(s["CTFBetaFac"])[:4])
        c.FP16Volume = _bool(opt("FP16Volume", "false"))
        c.WriteVolumeAsFP16 = _bool(opt("WriteVolumeAsFP16", "false"))
        c.ProjectionScaleFactor = float(opt("ProjectionScaleFactor", "1"))
        c.WBP = _bool(opt("WBP", "false"))
        c.DoseWeighting = _bool(opt("DoseWeighting", "false"))
        if c.DoseWeighting:
            c.AccumulatedDose = _floats(req("AccumulatedDose"))
        c.DownWeightTiltsForWBP = _bool(opt("DownWeightTiltsForWBP", "false"))
        c.SwitchCTFDirectionForIMOD = _bool(opt("SwitchCTFDirectionForIMOD", "false"))
        c.PhaseFlipOnly = _bool(opt("PhaseFlipOnly", "false"))
        c.WienerFilterNoiseLevel = float(opt("WienerFilterNoiseLevel", "0.1"))
        f = opt("WBPFilter", "")
        if f and f.lower() in WBP_FILTERS and f in (f.lower(), f.upper(), f.capitalize()):
            c.WBPFilter = WBP_FILTERS[f.lower()]
        c.CtfMode = _bool(req("CtfMode"))
        if c.CtfMode:
            c.CtfFile = req("CtfFile")
            c.Cs = float(req("Cs"))
            c.Voltage = float(req("Voltage"))
        c.BadPixelValue = float(req("BadPixelValue"))
        c.CorrectBadPixels = _bool(req("CorrectBadPixels"))
        pn = opt("ProjectionNormalization", "")
        if pn in ("STD", "std", "StandardDeviation"):
            c.ProjectionNormalization = 1
        elif pn in ("NONE", "none", "None"):
            c.ProjectionNormalization = 2
        m = _floats(opt("MagAnisotropy", ""))
        if len(m) >= 2:
            c.MagAnisotropy = (m[0], m[1])
        c.IgnoreZShiftForCTF = _bool(opt("IgnoreZShiftForCTF", "false"))
        c.CTFSliceThickness = float(opt("CTFSliceThickness", "50"))
        if subvolumes:
            c.SizeSubVol = int(float(req("SizeSubVol")))
            c.VoxelSizeSubVol = float(req("VoxelSizeSubVol"))
            c.MotiveList = req("MotiveList")
            c.SubVolPath = req("SubVolPath")
            c.ShiftInputFile = req("ShiftInputFile")
            c.BatchSize = int(float(req("BatchSize")))
            c.MaxShift = int(float(req("MaxShift")))
            c.NamingConvention = 1 if opt("NamingConvention", "") in ("TomoParticle", "Tomo_Particle") else 0
            c.ScaleMotivelistShift = float(req("ScaleMotivelistShift"))
            c.ScaleMotivelistPosition = float(req("ScaleMotivelistPosition"))
        if refine:
            c.SizeSubVol = int(float(req("SizeSubVol")))
            c.VoxelSizeSubVol = float(req("VoxelSizeSubVol"))
            c.MotiveList = req("MotiveList")
            c.Reference = req("Reference")
            c.MaxShift = int(float(req("MaxShift")))
            c.ShiftOutputFile = req("ShiftOutputFile")
            c.GroupMode = req("GroupMode")
            if c.GroupMode not in ("ByGroup", "MaxDistance", "MaxCount"):
                raise ValueError("GroupMode: ByGroup, MaxDistance or MaxCount expected")
            if c.GroupMode == "MaxDistance":
                c.MaxDistance = float(req("MaxDistance"))
            if c.GroupMode == "MaxCount":
                c.GroupSize = int(float(req("GroupSize")))
            c.CCMapFileName = opt("CCMapFileName", "")
            c.SpeedUpDistance = int(float(req("SpeedUpDistance")))
            c.ScaleMotivelistShift = float(req("ScaleMotivelistShift"))
            c.ScaleMotivelistPosition = float(req("ScaleMotivelistPosition"))
            c.MultiPeakDetection = _bool(req("MultiPeakDetection"))
            # ';'-separated lists; items of 3 characters or fewer are dropped
            # (utils/Config.cpp:449-475)
            refs = opt("SupportingReferences", "")
            if len(refs) > 3:
                c.SupportingReferences = [it for it in refs.split(";") if len(it) > 3]
                lists = req("SupportingMotiveLists")
                if len(lists) > 3:
                    c.SupportingMotiveLists = [it for it in lists.split(";") if len(it) > 3]
                c.MaxDistanceSupport = float(req("MaxDistanceSupport"))
        return c

    @classmethod
    def from_file(cls, path: str, subvolumes: bool = False, refine: bool = False) -> "EmSartConfig":
        with open(path) as f:
            return cls.from_text(f.read(), subvolumes, refine)


