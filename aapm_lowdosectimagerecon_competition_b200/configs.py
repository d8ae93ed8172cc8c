"""Seeded synthetic workloads standing in for the AAPM low-dose CT data.

The reference reconstructs AAPM DICOM-CT-PD projections (not available here);
these generators reproduce the workload shapes: scanner geometry, image grid,
slice and view counts, and the value ranges of attenuation images (mm^-1).
Seeds use numpy's PCG64 (numpy.random.default_rng).

  c1  256^2 x 1 slice, 1.0 mm, 984 views, 888 channels, sid 541, sdd 949
  c2  512^2 x 64 slices, 0.7 mm, 2304 views, 736 channels at 1.2858 mm, sid 595, sdd 1085.6
  c3  c2 geometry, 128 slices, 24 subsets x 10 iterations, FISTA + non-negativity,
      log of Poisson counts at I0 = 1.5e5 photons per ray
  c4  32 instances: side {256,384,512,768}, slices 8..96, views 720..2304, 736 channels
"""
import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Scan:
    XN: int
    YN: int
    dx: float
    SLN: int
    PN: int            # views over 360 degrees
    DNU: int
    sid: float
    sdd: float
    detCellWidth: float  # channel pitch at the detector (mm)
    detCntIdx: float     # 1-based central channel index, as in the reference's cfg
    numOfOS: int = 1
    numOfIter: int = 1
    useFISTA: int = 1
    nonneg: int = 0
    I0: float = 0.0

    def conf(self):
        """The reference's conf struct (AAPM_script/ConvertToReconConf.m:21-34)."""
        return {"recon": {"XN": self.XN, "YN": self.YN, "dx": self.dx}, "SLN": self.SLN,
                "acq": {"sid": self.sid, "sdd": self.sdd, "DNU": self.DNU, "PN": self.PN,
                        "detCellWidth": self.detCellWidth, "detCntIdx": self.detCntIdx}}

    def angles(self, PN=None):
        """Equiangular views over 360 degrees, float32 (PN,)."""
        PN = self.PN if PN is None else PN
        return (np.arange(PN, dtype=np.float64) * (2.0 * math.pi / PN)).astype(np.float32)

    def hangs(self, PN=None):
        """Per-slice view angles (PN, SLN) -- all slices share the list."""
        a = self.angles(PN)
        return np.repeat(a[:, None], self.SLN, axis=1)

    def rebinned_hangs(self, spacing=36, BV=0.0):
        """Per-slice view angles (PN, SLN) as helical rebinning leaves them:
        slice z starts at raw view 1 + floor(spacing * z) and its view ib has
        angle mod((start + ib - 1) * delta + BV, 2 pi) in float32
        (AAPM_script/HelicalToFanFunc_mex.cpp:77-81) -- one grid, circularly
        shifted per slice, different in the last bits from slice to slice.
        A non-integer spacing gives the irregular starts of slices at
        linspace positions (reconscript.m:22)."""
        f = np.float32
        delta, twopi = f(2.0 * math.pi / self.PN), f(2.0 * math.pi)
        starts = np.floor(spacing * np.arange(self.SLN)).astype(np.int64)
        i = (np.arange(self.PN)[:, None] + starts[None, :]).astype(np.float32)
        lam = (i * delta).astype(np.float32) + f(BV)
        # the reference's repeated float subtraction of 2 pi
        while True:
            over = lam > twopi
            if not over.any():
                break
            lam = np.where(over, (lam - twopi).astype(np.float32), lam)
        return lam.astype(np.float32)

    def circular_mask(self):
        """Disk mask of AAPM_script/reconscript.m:28-38 (radius 1.3 of the half
        width, i.e. nearly everything), as (YN, XN) bytes."""
        ii = np.arange(1, self.XN + 1, dtype=np.float64)[None, :]
        jj = np.arange(1, self.YN + 1, dtype=np.float64)[:, None]
        r = np.sqrt(((ii - 0.5 - self.XN / 2) / (self.XN / 2)) ** 2 +
                    ((jj - 0.5 - self.YN / 2) / (self.YN / 2)) ** 2)
        return (r < 1.3).astype(np.uint8)


def c1():
    return Scan(XN=256, YN=256, dx=1.0, SLN=1, PN=984, DNU=888, sid=541.0, sdd=949.0,
                detCellWidth=1.0239, detCntIdx=(888 + 1) / 2.0, numOfOS=8, numOfIter=5)


def c2(SLN=64):
    return Scan(XN=512, YN=512, dx=0.7, SLN=SLN, PN=2304, DNU=736, sid=595.0, sdd=1085.6,
                detCellWidth=1.2858, detCntIdx=368.5)


def c3(SLN=128):
    s = c2(SLN)
    s.numOfOS, s.numOfIter, s.useFISTA, s.nonneg, s.I0 = 24, 10, 1, 1, 1.5e5
    return s


def c4_instances(n=32, seed=4):
    """Config-4 size distribution: (N, SLN, PN) per instance."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(rng.choice([256, 384, 512, 768]))
        Z = int(rng.integers(8, 97))
        P = int(rng.integers(720, 2305))
        out.append((N, Z, P))
    return out


def scaled(scan, XN=None, SLN=None, PN=None, DNU=None):
    """A smaller copy of `scan` with the same field of view (for tests)."""
    s = dataclasses.replace(scan)
    if XN is not None:
        s.dx = scan.dx * scan.XN / XN
        s.XN = s.YN = XN
    if DNU is not None:
        s.detCellWidth = scan.detCellWidth * scan.DNU / DNU
        s.DNU = DNU
        s.detCntIdx = (DNU + 1) / 2.0
    if SLN is not None:
        s.SLN = SLN
    if PN is not None:
        s.PN = PN
    return s


# ---------------------------------------------------------------- phantoms

def ellipse_phantom_2d(scan, n=10, seed=1):
    """Water disk (0.02 / mm) with n random ellipses of mu in [0, 0.04] / mm,
    float32 (YN, XN, 1)."""
    rng = np.random.default_rng(seed)
    N = scan.XN
    c = (np.arange(N) - (N - 1) / 2.0) * scan.dx
    X, Y = np.meshgrid(c, c, indexing="xy")
    R = 0.43 * N * scan.dx
    img = np.where(X ** 2 + Y ** 2 <= R ** 2, 0.02, 0.0)
    for _ in range(n):
        cx, cy = rng.uniform(-0.6, 0.6, 2) * R
        a, b = rng.uniform(0.04, 0.3, 2) * R
        th = rng.uniform(0, math.pi)
        mu = rng.uniform(0.0, 0.04)
        xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
        yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
        img = np.where((xr / a) ** 2 + (yr / b) ** 2 <= 1.0, mu, img)
    return img.astype(np.float32)[:, :, None]


def ellipsoid_phantom_3d(scan, n=10, seed=2):
    """Water cylinder with n random ellipsoids, float32 (YN, XN, SLN); the
    slice spacing is taken equal to dx."""
    rng = np.random.default_rng(seed)
    N, Z = scan.XN, scan.SLN
    c = (np.arange(N) - (N - 1) / 2.0) * scan.dx
    zc = (np.arange(Z) - (Z - 1) / 2.0) * scan.dx
    X, Y = np.meshgrid(c, c, indexing="xy")
    R = 0.43 * N * scan.dx
    body = (X ** 2 + Y ** 2 <= R ** 2)
    img = np.repeat(np.where(body, 0.02, 0.0)[:, :, None], Z, axis=2).astype(np.float32)
    H = max(Z * scan.dx, scan.dx)
    for _ in range(n):
        cx, cy = rng.uniform(-0.6, 0.6, 2) * R
        cz = rng.uniform(-0.5, 0.5) * H
        a, b = rng.uniform(0.04, 0.3, 2) * R
        cc = rng.uniform(0.2, 0.8) * H
        th = rng.uniform(0, math.pi)
        mu = rng.uniform(0.0, 0.04)
        xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
        yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
        q2 = (xr / a) ** 2 + (yr / b) ** 2
        zz = ((zc - cz) / cc) ** 2
        inside = q2[:, :, None] + zz[None, None, :] <= 1.0
        img[inside] = mu
    return img


def phantom(scan, seed=2):
    return ellipse_phantom_2d(scan, seed=seed) if scan.SLN == 1 else ellipsoid_phantom_3d(scan, seed=seed)


def poisson_log(prj, I0, seed=3):
    """y = -ln(max(n, 1) / I0), n ~ Poisson(I0 exp(-prj)) (numpy, float32)."""
    rng = np.random.default_rng(seed)
    lam = I0 * np.exp(-np.asarray(prj, np.float64))
    n = rng.poisson(lam)
    return (-np.log(np.maximum(n, 1) / I0)).astype(np.float32)
