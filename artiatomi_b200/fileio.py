"""EM and MRC files, marker files and CTF files as EmSART reads and writes them.

The layouts are the reference's (they define the files users already have):

* EM (src/EmTools/FileIO/EmHeader.h): a 512-byte header -- machine coding,
  two unused bytes, data type, DimX/DimY/DimZ (int32), an 80-byte comment,
  40 int32 parameters (voltage, Cs, ..., ObjectPixelSize at factor 1000 nm,
  ..., IsNewHeaderFormat, AlignmentScore, BeamDeclination, MarkerOffset,
  MagAnisotropyFactor/Angle, ImageSizeX/Y) and 256 bytes of user data --
  then the data with x fastest. Data types: 1 uint8, 2 int16, 4 int32,
  5 float32, 8 complex64, 9 float64, 10 float16 (EMDATATYPE_HALF). Machine
  codes 3 (SGI) and 5 (Mac) are big-endian, the others little-endian.
* MRC (src/EmTools/FileIO/mrcHeader.h): a 1024-byte header (NX, NY, NZ,
  MODE, starts, MX/MY/MZ, cell lengths in Angstrom, angles, MAPC/MAPR/MAPS,
  min/max/mean, ISPG, NSYMBT, NEXT, ..., CMAP "MAP ", STAMP, RMS, 10 labels)
  plus NEXT bytes of extended header. Modes: 0 uint8 (int8 when IMODFlags
  bit 0 is set), 1 int16, 2 float32, 4 complex64, 6 uint16, 12 and 64
  float16 (64 is the reference's MRCMODE_HALF). Pixel size (nm) =
  Xlen / NX / 10.
* Marker file (src/EmTools/FileIO/MarkerFile.{h,cpp}): an EM float file of
  10 x projections x markers; item i of projection p and marker m is
  data[m][p][i] with items tilt angle, x/y coordinate, deviation, x/y shift,
  projected x/y, magnification, psi. A projection is used when the
  reference marker's coordinates are > -1.
* CTF file (src/EmTools/FileIO/CtfFile.cpp): an EM float file of
  projections columns; row 1 holds the minimum defocus, row 2 the maximum
  (nm), row 4 the astigmatism angle (rad).
* Motive list (src/EmTools/FileIO/MotiveListe.h, MotiveList.cpp): an EM
  float file of 20 x particles (cc, x/y click, particle nr, tomogram nr,
  particle nr in tomogram, wedge, x/y/z coordinate, x/y/z shift, shifts
  before, phi, psi, theta, class); coordinates and shifts are scaled by the
  binning factors at read.
* Shift file (src/EmTools/FileIO/ShiftFile.cpp): an EM float file of
  motives x projections x 2; the extra shift of (projection, motive) is the
  negated stored pair.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

# ----------------------------------------------------------------------- EM
EM_DTYPES = {1: np.uint8, 2: np.int16, 4: np.int32, 5: np.float32, 8: np.complex64, 9: np.float64, 10: np.float16}
EM_PARAMS = ["Voltage", "Cs", "Aperture", "Magnification", "PostMagnification", "ExposureTime", "ObjectPixelSize",
             "Microscope", "Pixelsize", "CCDArea", "Defocus", "Astigmatism", "AstigmatismAngle", "FocusIncrement",
             "CountsPerElectron", "Intensity", "EnergySlitwidth", "EnergyOffset", "Tiltangle", "Tiltaxis",
             "IsNewHeaderFormat", "AlignmentScore", "BeamDeclination", "MarkerOffset", "MagAnisotropyFactor",
             "MagAnisotropyAngle", "ImageSizeX", "ImageSizeY"]
EM_FLOAT_PARAMS = {"AlignmentScore", "BeamDeclination", "MagAnisotropyFactor", "MagAnisotropyAngle"}


def _em_header_dtype(endian: str) -> np.dtype:
    fields = [("MachineCoding", "i1"), ("NotUsed1", "i1"), ("NotUsed2", "i1"), ("DataType", "i1"),
              ("DimX", endian + "i4"), ("DimY", endian + "i4"), ("DimZ", endian + "i4"), ("Comment", "S80")]
    for p in EM_PARAMS:
        fields.append((p, endian + ("f4" if p in EM_FLOAT_PARAMS else "i4")))
    fields += [("Fillup1", endian + "i4", (12,)), ("Username", "S20"), ("Date", "S8"), ("Fillup2", "S228")]
    dt = np.dtype(fields)
    assert dt.itemsize == 512
    return dt


def read_em(path: str):
    """(array [z][y][x], header record)."""
    with open(path, "rb") as f:
        raw = f.read(512)
        machine = raw[0]
        endian = ">" if machine in (3, 5) else "<"
        hdr = np.frombuffer(raw, _em_header_dtype(endian))[0]
        dt = EM_DTYPES.get(int(hdr["DataType"]))
        if dt is None:
            raise ValueError(f"{path}: unsupported EM data type {int(hdr['DataType'])}")
        nx, ny, nz = int(hdr["DimX"]), int(hdr["DimY"]), int(hdr["DimZ"])
        data = np.fromfile(f, dtype=np.dtype(dt).newbyteorder(endian), count=nx * ny * nz)
    if data.size != nx * ny * nz:
        raise ValueError(f"{path}: file shorter than its header says")
    return data.astype(np.dtype(dt).newbyteorder("=")).reshape(nz, ny, nx), hdr


def write_em(path: str, data: np.ndarray, header: dict | None = None) -> None:
    """Little-endian (PC) EM file; data [z][y][x] (or [y][x]). header: extra
    fields of the EM header by name (e.g. ObjectPixelSize)."""
    a = np.asarray(data)
    if a.ndim == 2:
        a = a[None]
    codes = {np.dtype(v): k for k, v in EM_DTYPES.items()}
    if a.dtype not in codes:
        raise ValueError(f"unsupported dtype {a.dtype} for EM")
    hdr = np.zeros(1, _em_header_dtype("<"))[0]
    hdr["MachineCoding"] = 6
    hdr["DataType"] = codes[a.dtype]
    hdr["DimX"], hdr["DimY"], hdr["DimZ"] = a.shape[2], a.shape[1], a.shape[0]
    for k, v in (header or {}).items():
        hdr[k] = v
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes())


# ---------------------------------------------------------------------- MRC
MRC_DTYPES = {0: np.uint8, 1: np.int16, 2: np.float32, 4: np.complex64, 6: np.uint16, 12: np.float16,
              64: np.float16}


def _mrc_header_dtype(endian: str) -> np.dtype:
    e = endian
    dt = np.dtype([("NX", e + "i4"), ("NY", e + "i4"), ("NZ", e + "i4"), ("MODE", e + "i4"),
                   ("NXSTART", e + "i4"), ("NYSTART", e + "i4"), ("NZSTART", e + "i4"),
                   ("MX", e + "i4"), ("MY", e + "i4"), ("MZ", e + "i4"),
                   ("Xlen", e + "f4"), ("Ylen", e + "f4"), ("Zlen", e + "f4"),
                   ("ALPHA", e + "f4"), ("BETA", e + "f4"), ("GAMMA", e + "f4"),
                   ("MAPC", e + "i4"), ("MAPR", e + "i4"), ("MAPS", e + "i4"),
                   ("AMIN", e + "f4"), ("AMAX", e + "f4"), ("AMEAN", e + "f4"),
                   ("ISPG", e + "u2"), ("NSYMBT", e + "u2"), ("NEXT", e + "i4"), ("CREATEID", e + "u2"),
                   ("EXTRA", "S30"), ("NINT", e + "u2"), ("NREAL", e + "u2"), ("EXTRA2", "S20"),
                   ("IMODStamp", e + "i4"), ("IMODFlags", e + "i4"), ("IDTYPE", e + "u2"), ("LENS", e + "u2"),
                   ("ND1", e + "u2"), ("ND2", e + "u2"), ("VD1", e + "u2"), ("VD2", e + "u2"),
                   ("TILTANGLES", e + "f4", (6,)), ("XORIGIN", e + "f4"), ("YORIGIN", e + "f4"),
                   ("ZORIGIN", e + "f4"), ("CMAP", "S4"), ("STAMP", e + "u4"), ("RMS", e + "f4"),
                   ("NLABL", e + "i4"), ("LABELS", "S80", (10,))])
    assert dt.itemsize == 1024
    return dt


def read_mrc(path: str):
    """(array [z][y][x], header record)."""
    with open(path, "rb") as f:
        raw = f.read(1024)
        stamp = raw[212]  # MACHST byte 0: 0x44 little-endian, 0x11 big-endian
        endian = ">" if stamp == 0x11 else "<"
        hdr = np.frombuffer(raw, _mrc_header_dtype(endian))[0]
        mode = int(hdr["MODE"])
        dt = MRC_DTYPES.get(mode)
        if dt is None:
            raise ValueError(f"{path}: unsupported MRC mode {mode}")
        if mode == 0 and int(hdr["IMODStamp"]) == 1146047817 and (int(hdr["IMODFlags"]) & 1):
            dt = np.int8
        f.seek(1024 + max(0, int(hdr["NEXT"])))
        nx, ny, nz = int(hdr["NX"]), int(hdr["NY"]), int(hdr["NZ"])
        data = np.fromfile(f, dtype=np.dtype(dt).newbyteorder(endian), count=nx * ny * nz)
    if data.size != nx * ny * nz:
        raise ValueError(f"{path}: file shorter than its header says")
    return data.astype(np.dtype(dt).newbyteorder("=")).reshape(nz, ny, nx), hdr


def mrc_pixel_size_nm(hdr) -> float:
    nx = int(hdr["NX"])
    return float(hdr["Xlen"]) / nx / 10.0 if nx > 0 and float(hdr["Xlen"]) > 0 else 1.0


def write_mrc(path: str, data: np.ndarray, pixel_size_nm: float = 1.0, half_mode: int = 64) -> None:
    """MRC file as MRCFile::SetHeaderData writes it (cell lengths = dims x
    pixel size x 10 Angstrom, axes X/Y/Z, CMAP "MAP "); float16 data is written
    with mode `half_mode` (64: the reference's MRCMODE_HALF, 12: the MRC2014
    code)."""
    a = np.asarray(data)
    if a.ndim == 2:
        a = a[None]
    modes = {np.dtype(np.uint8): 0, np.dtype(np.int16): 1, np.dtype(np.float32): 2, np.dtype(np.complex64): 4,
             np.dtype(np.uint16): 6, np.dtype(np.float16): half_mode}
    if a.dtype not in modes:
        raise ValueError(f"unsupported dtype {a.dtype} for MRC")
    hdr = np.zeros(1, _mrc_header_dtype("<"))[0]
    nz, ny, nx = a.shape
    hdr["NX"], hdr["NY"], hdr["NZ"], hdr["MODE"] = nx, ny, nz, modes[a.dtype]
    hdr["MX"], hdr["MY"], hdr["MZ"] = nx, ny, nz
    hdr["Xlen"], hdr["Ylen"], hdr["Zlen"] = nx * pixel_size_nm * 10.0, ny * pixel_size_nm * 10.0, nz * pixel_size_nm * 10.0
    hdr["ALPHA"] = hdr["BETA"] = hdr["GAMMA"] = 90.0
    hdr["MAPC"], hdr["MAPR"], hdr["MAPS"] = 1, 2, 3
    if a.size and not np.iscomplexobj(a):
        af = a.astype(np.float64)
        hdr["AMIN"], hdr["AMAX"], hdr["AMEAN"] = af.min(), af.max(), af.mean()
        hdr["RMS"] = af.std()
    hdr["CMAP"] = b"MAP "
    hdr["STAMP"] = 0x00004444
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes())


# ----------------------------------------------------------------- volumes
def write_volume(path: str, vol: np.ndarray, pixel_size_nm: float, voxel_size: float = 1.0) -> None:
    """The reconstruction's output file by extension, as EmSart.cpp:694-813:
    .em -> EM (ObjectPixelSize = pixel size x voxel size x 1000), .mrc/.rec
    -> MRC (cell = dims x pixel size x voxel size x 10 Angstrom), anything
    else -> raw: DimX, DimY, DimZ (int32), maximum (float32), data."""
    if path.rfind(".em") >= 0:
        write_em(path, vol, {"ObjectPixelSize": int(pixel_size_nm * voxel_size * 1000)})
    elif path.rfind(".mrc") >= 0 or path.rfind(".rec") >= 0:
        write_mrc(path, vol, pixel_size_nm * voxel_size)
    else:
        a = np.ascontiguousarray(vol, np.float32)
        with open(path, "wb") as f:
            np.array([a.shape[2], a.shape[1], a.shape[0]], "<i4").tofile(f)
            np.array([a.max() if a.size else -999999.0], "<f4").tofile(f)
            a.astype("<f4").tofile(f)


def read_stack(path: str):
    """Tilt series (projections [n][H][W]) and its pixel size in nm."""
    if path.rfind(".em") >= 0 and not path.endswith((".mrc", ".st", ".rec")):
        data, hdr = read_em(path)
        ps = int(hdr["ObjectPixelSize"]) / 1000.0
        return data, (ps if ps > 0 else 1.0)
    data, hdr = read_mrc(path)
    return data, mrc_pixel_size_nm(hdr)


# --------------------------------------------------------------- markers
MFI = dict(TiltAngle=0, X_Coordinate=1, Y_Coordinate=2, DevOfMark=3, X_Shift=4, Y_Shift=5,
           ProjectedCoordinateX=6, ProjectedCoordinateY=7, Magnification=8, RotationPsi=9)


@dataclass
class MarkerData:
    """Marker file contents: items[marker][projection][10]."""

    items: np.ndarray
    ref_marker: int = 0
    mag_anisotropy: tuple | None = None  # (factor, angle deg, image x, image y) of the new header format

    @property
    def projection_count(self) -> int:
        return int(self.items.shape[1])

    def item(self, name: str, marker: int = 0) -> np.ndarray:
        return self.items[marker, :, MFI[name]].astype(np.float32)

    def good(self) -> np.ndarray:
        """MarkerFile::CheckIfProjIndexIsGood: the reference marker is clicked."""
        r = self.ref_marker
        return (self.items[r, :, 1] > -1) & (self.items[r, :, 2] > -1)

    def markers(self):
        """Alignment of each projection (marker 0's items, as Projection reads them)."""
        from .emsart import Markers

        return Markers(self.item("TiltAngle"), self.item("X_Shift"), self.item("Y_Shift"),
                       self.item("Magnification"), self.item("RotationPsi"))


def read_markers(path: str, ref_marker: int = 0) -> MarkerData:
    data, hdr = read_em(path)
    if data.shape[2] != 10:
        raise ValueError(f"{path}: not a marker file (DimX = {data.shape[2]}, expected 10)")
    mag = None
    if int(hdr["IsNewHeaderFormat"]):
        mag = (float(hdr["MagAnisotropyFactor"]), float(hdr["MagAnisotropyAngle"]), int(hdr["ImageSizeX"]),
               int(hdr["ImageSizeY"]))
    return MarkerData(data.astype(np.float32), ref_marker, mag)


def write_markers(path: str, items: np.ndarray) -> None:
    """items[marker][projection][10] as an EM float file."""
    write_em(path, np.ascontiguousarray(items, np.float32))


# -------------------------------------------------------------------- CTF
def read_ctf(path: str) -> np.ndarray:
    """Defocus table [projection][3]: minimum and maximum defocus (nm) and the
    astigmatism angle (deg), the layout esb_reconstructor_create takes."""
    data, _ = read_em(path)
    d = data[0].astype(np.float32)  # [row][projection]
    out = np.stack([d[1], d[2], (d[4] * np.float32(180.0) / np.float32(np.pi)).astype(np.float32)], 1)
    return np.ascontiguousarray(out, np.float32)


def write_ctf(path: str, defocus_min, defocus_max, astig_rad) -> None:
    n = len(defocus_min)
    d = np.zeros((5, n), np.float32)
    d[1], d[2], d[4] = defocus_min, defocus_max, astig_rad
    write_em(path, d[None])


# ------------------------------------------------------------ motive list
MOTL_FIELDS = ["ccCoeff", "xCoord", "yCoord", "partNr", "tomoNr", "partNrInTomo", "wedgeIdx", "x_Coord", "y_Coord",
               "z_Coord", "x_Shift", "y_Shift", "z_Shift", "x_ShiftBefore", "y_ShiftBefore", "z_ShiftBefore", "phi",
               "psi", "theta", "classNo"]


def read_motive_list(path: str, scale_position: float = 1.0, scale_shift: float = 1.0) -> np.ndarray:
    """Particles [n][20] (MotiveList::GetAt: click coordinates and x/y/z
    coordinates times scale_position, x/y/z shifts times scale_shift)."""
    data, _ = read_em(path)
    if data.shape[2] != 20:
        raise ValueError(f"{path}: not a motive list (DimX = {data.shape[2]}, expected 20)")
    m = data.reshape(-1, 20).astype(np.float32).copy()
    for k in (1, 2, 7, 8, 9):
        m[:, k] *= np.float32(scale_position)
    for k in (10, 11, 12):
        m[:, k] *= np.float32(scale_shift)
    return m


def write_motive_list(path: str, particles: np.ndarray) -> None:
    write_em(path, np.ascontiguousarray(particles, np.float32).reshape(1, -1, 20))


def index_coding(particle: np.ndarray, tomo_particle: bool = False) -> str:
    """motive::GetIndexCoding: the particle number (or tomogram_particle),
    formatted as a C++ stream formats a float."""
    def g(v):
        return "%g" % float(np.float32(v))

    return f"{g(particle[4])}_{g(particle[5])}" if tomo_particle else g(particle[3])


def read_shift_file(path: str) -> np.ndarray:
    """Extra shifts [projection][motive][2] (ShiftFile::operator(): negated)."""
    data, _ = read_em(path)  # [2][projections][motives]
    return np.ascontiguousarray(-np.moveaxis(data.astype(np.float32), 0, -1))


def write_shift_file(path: str, stored: np.ndarray) -> None:
    """stored [2][projections][motives] as the file holds it."""
    write_em(path, np.ascontiguousarray(stored, np.float32))


def exists(path: str) -> bool:
    return bool(path) and os.path.exists(path)
