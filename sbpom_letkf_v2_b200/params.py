"""Run-time parameter set of the analysis step.

The reference fixes every knob at compile time as a Fortran PARAMETER in
``letkf/run/src/common_setting.f90`` (lines 15-131).  Here they become one
run-time record, mirrored field for field by ``struct sbletkf_params`` in
``include/sbletkf.h``.  Defaults are the reference's values except the sizes,
which belong to the workload.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

DA_LETKF, DA_LPF, DA_LPFGM = 1, 2, 3          # iswitch_da, common_setting.f90:65
RM_SR, RM_MR = 0, 1                           # RM, common_setting.f90:82
PREC_FP64, PREC_MIXED = 0, 1
F32, F64 = 0, 1

# element ids, common_setting.f90:56-60
ID_U_OBS, ID_V_OBS, ID_T_OBS, ID_Z_OBS, ID_S_OBS = 2819, 2820, 3073, 2567, 3332

#: cutoff / scale ratio of the Gaussian localization, common_setting.f90:97-98
CUTOFF_RATIO = 2.0 * math.sqrt(10.0 / 3.0)


class CParams(ctypes.Structure):
    """ctypes image of ``struct sbletkf_params``."""

    _fields_ = [
        ("nmem", ctypes.c_int32), ("nlon", ctypes.c_int32), ("nlat", ctypes.c_int32),
        ("nlev", ctypes.c_int32), ("nv3d", ctypes.c_int32), ("nv2d", ctypes.c_int32),
        ("iv3d_t", ctypes.c_int32), ("iv3d_s", ctypes.c_int32),
        ("iswitch_da", ctypes.c_int32), ("nmonte", ctypes.c_int32), ("rm", ctypes.c_int32),
        ("dp", ctypes.c_int32), ("sr_textbook", ctypes.c_int32), ("roff", ctypes.c_int32),
        ("id_z_obs", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("max_sweeps", ctypes.c_int32),
        ("iv3d_u", ctypes.c_int32), ("iv3d_v", ctypes.c_int32), ("iv2d_z", ctypes.c_int32),
        ("cov_infl_mul", ctypes.c_double), ("cov_infl_gm", ctypes.c_double),
        ("alpha_rtpp", ctypes.c_double), ("alpha_rtps", ctypes.c_double),
        ("sigma_obs", ctypes.c_double), ("sigma_obsv", ctypes.c_double),
        ("dist_zero", ctypes.c_double), ("dist_zerov", ctypes.c_double),
        ("tmin", ctypes.c_double), ("tmax", ctypes.c_double),
        ("smin", ctypes.c_double), ("smax", ctypes.c_double),
        ("re", ctypes.c_double), ("pi", ctypes.c_double),
        ("jacobi_tol", ctypes.c_double), ("tc_max_cand", ctypes.c_double),
        ("jacobi_stop", ctypes.c_double), ("reserved_d", ctypes.c_double * 1),
    ]


@dataclasses.dataclass
class LETKFParams:
    """The analysis-step knobs of ``common_setting.f90``.

    ``dist_zero``/``dist_zerov`` default to ``2*sqrt(10/3)`` times the
    localization scales (common_setting.f90:97-98) when left as ``None``.
    """

    nmem: int = 128                 # :36
    nlon: int = 1442                # :37
    nlat: int = 562                 # :38
    nlev: int = 75                  # :39
    nv3d: int = 4                   # :40  (u, v, t, s)
    nv2d: int = 3                   # :41  (zeta, ubar, vbar)
    iv3d_t: int = 2                 # :44 (1-based 3 -> 0-based 2)
    iv3d_s: int = 3                 # :45
    iswitch_da: int = DA_LETKF      # :65
    nmonte: int = 100               # :79
    rm: int = RM_MR                 # :82
    dp: bool = True                 # :85
    sr_textbook: bool = False       # reference SR offset quirk, common_lpfgm.f90:115-117
    roff: bool = True               # :129
    id_z_obs: int = ID_Z_OBS        # :59
    precision: int = PREC_FP64
    max_sweeps: int = 40
    iv3d_u: int = 0                 # :42 (1-based 1 -> 0-based 0)
    iv3d_v: int = 1                 # :43
    iv2d_z: int = 0                 # :46
    cov_infl_mul: float = 1.0       # :71
    cov_infl_gm: float = 1.0        # :89
    alpha_rtpp: float = 0.9         # :74
    alpha_rtps: float = 0.0         # :75
    sigma_obs: float = 300.0e3      # :94
    sigma_obsv: float = 100.0       # :95
    dist_zero: float | None = None  # :97
    dist_zerov: float | None = None  # :98
    tmin: float = -1.8              # :130
    tmax: float = 50.0
    smin: float = 25.0              # :131
    smax: float = 50.0
    re: float = 6371.3e3            # :28
    pi: float = 4.0 * math.atan(1.0)  # :27
    jacobi_tol: float = 0.0         # 0 -> library default (k * eps FP64, 1e-8 mixed)
    tc_max_cand: float = 0.0        # mixed path: FP64 Gram above this many box candidates (0 -> 12288)
    jacobi_stop: float = 0.0        # end the eigensolve after a sweep with no relative rotation above this (0 -> 1e-10 FP64, 1e-5 mixed)

    def __post_init__(self):
        if self.dist_zero is None:
            self.dist_zero = CUTOFF_RATIO * self.sigma_obs
        if self.dist_zerov is None:
            self.dist_zerov = CUTOFF_RATIO * self.sigma_obsv

    def replace(self, **kw) -> "LETKFParams":
        """Copy with fields changed; cutoffs follow the scales unless given."""
        d = dataclasses.asdict(self)
        if "sigma_obs" in kw and "dist_zero" not in kw:
            d["dist_zero"] = None
        if "sigma_obsv" in kw and "dist_zerov" not in kw:
            d["dist_zerov"] = None
        d.update(kw)
        return LETKFParams(**d)

    def validate(self) -> None:
        if self.nmem < 2 or self.nmem > 128:
            raise ValueError(f"nmem={self.nmem}: supported range is 2..128")
        if self.nlev < 1 or self.nlon < 2 or self.nlat < 2:
            raise ValueError("grid sizes must be nlev>=1, nlon>=2, nlat>=2")
        if self.nv3d < 0 or self.nv2d < 0 or self.nv3d + self.nv2d > 8:
            raise ValueError("nv3d+nv2d must be <= 8")
        if self.iswitch_da not in (DA_LETKF, DA_LPF, DA_LPFGM):
            raise ValueError(f"Incorrect iswitch_da ==> {self.iswitch_da}")
        if self.rm not in (RM_SR, RM_MR):
            raise ValueError(f"Incorrect RM ==> {self.rm}")
        if self.cov_infl_mul <= 0 or self.cov_infl_gm <= 0:
            raise ValueError("inflation factors must be > 0")
        if self.sigma_obs <= 0:
            raise ValueError("sigma_obs must be > 0")
        if self.nmonte < 1:
            raise ValueError("nmonte must be >= 1")

    def to_c(self) -> CParams:
        c = CParams()
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        return c
