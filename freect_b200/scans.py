"""Seeded synthetic helical scans with the scanner shapes of the benchmark
configurations (there are no measured datasets in this project).

Geometry conventions (the ones the reference's rebin and backprojection
invert, see k_synth.cu): reading v has tube angle angle0 - v*2*pi/P and table
position z0 - v*feed/P, with the table centred on z = 0; raw frames are
[reading][row][channel] like ReconstructionMachine::AllocateKeyArrays
(ReconstructionMachine.cu:88-93).

Workloads:
  small     672 ch x 16 rows (0.6 mm), 1160 views/rot, 3 rotations, pitch 1,
            head-like ellipsoid phantom, I0 1e5, 256^2 x 16 slices @ 1 mm,
            250 mm FOV, Ram-Lak (generate_filter c = a = 1).
  rows64    888 ch x 64 rows (0.625 mm), 984 views/rot, 10 rotations,
            39.37 mm/rot, 320x240 mm water cylinder + 20 seeded ellipsoids
            (HU U[-1000, 1500]), I0 2e5, 512^2 x 300 slices @ 1 mm, 360 mm FOV,
            Shepp-Logan kernel. Fan spacing 2 asin(250/541)/887 rad and central
            channel 443.75 are chosen here (a 500 mm acquisition FOV).
  tiny/...  reduced shapes for tests.
"""
import dataclasses
import math

import numpy as np

from . import abi_types as T

MU_WATER = 0.019  # 1/mm


def hu_to_mu(hu):
    return MU_WATER * (1.0 + hu / 1000.0)


@dataclasses.dataclass
class ScanSpec:
    name: str
    sid: float
    sdd: float
    nch: int
    dbeta: float          # fan angle increment (rad)
    c0: float             # central channel
    nr: int
    row_iso: float        # row width at isocentre (mm)
    P: int                # readings per rotation
    rotations: float
    feed: float           # table feed per rotation (mm)
    i0: float
    nx: int
    ny: int
    fov: float
    slice_thickness: float
    slice_pitch: float
    n_slices: int
    window: int = T.FILTER_REFERENCE
    phantom: str = "head"
    seed: int = 0
    n_random: int = 0
    angle0: float = 0.0
    ffs_mode: int = T.FFS_NONE

    @property
    def V(self):
        return int(round(self.P * self.rotations))

    @property
    def dcol(self):
        return self.dbeta * self.sdd

    @property
    def drow(self):
        return self.row_iso * self.sdd / self.sid

    def views(self):
        """tube angles and table positions (float32, like RawDataSet's floats)"""
        v = np.arange(self.V, dtype=np.float64)
        tube = self.angle0 - v * (2 * math.pi / self.P)
        z0 = 0.5 * (self.V - 1) * self.feed / self.P
        table = z0 - v * self.feed / self.P
        return tube.astype(np.float32), table.astype(np.float32)

    def synth(self, i0=None, seed=None):
        s = T.SynthScan()
        s.n_readings, s.rows, s.channels, s.readings_per_rotation = self.V, self.nr, self.nch, self.P
        s.sid, s.sdd, s.dcol, s.drow = self.sid, self.sdd, self.dcol, self.drow
        s.central_channel = self.c0
        tube, table = self.views()
        s.angle0 = float(tube[0])
        s.dangle = -2 * math.pi / self.P
        s.z0 = 0.5 * (self.V - 1) * self.feed / self.P
        s.dz = -self.feed / self.P
        s.i0 = self.i0 if i0 is None else i0
        s.seed = (self.seed * 0x9E3779B97F4A7C15 + 12345) & 0xFFFFFFFFFFFFFFFF if seed is None else seed
        s.ffs_mode = self.ffs_mode
        return s

    def meta(self):
        m = T.ScanMeta()
        m.total_num_projections = self.V
        m.projections_per_rotation = self.P
        m.detector_channels = self.nch
        m.detector_rows = self.nr
        m.detector_transverse_spacing = self.dcol
        m.detector_axial_spacing = self.drow
        m.detector_central_channel = self.c0
        m.detector_central_row = (self.nr - 1) / 2.0
        m.dist_source_to_isocenter = self.sid
        m.dist_source_to_detector = self.sdd
        m.ffs_mode = self.ffs_mode
        m.anode_angle = 0.0
        return m

    def recon_config(self):
        rp = T.ReconConfig()
        rp.raw_data_dir = b"synthetic"
        rp.output_dir = b"."
        rp.output_file = b"reconstruction.dat"
        start = -0.5 * (self.n_slices - 1) * self.slice_pitch
        rp.start_pos = start
        rp.end_pos = start + (self.n_slices - 0.5) * self.slice_pitch
        rp.recon_fov = self.fov
        rp.slice_thickness = self.slice_thickness
        rp.slice_pitch = self.slice_pitch
        rp.nx, rp.ny = self.nx, self.ny
        rp.recon_kernel = self.window
        rp.x_origin = rp.y_origin = 0.0
        rp.tube_angle_offset = 0.0
        rp.adaptive_filtration_s = 0.0
        return rp

    def ellipsoids(self):
        return make_phantom(self)


def _E(cx, cy, cz, ax, ay, az, phi, mu):
    e = T.Ellipsoid()
    e.cx, e.cy, e.cz, e.ax, e.ay, e.az, e.phi, e.mu = cx, cy, cz, ax, ay, az, phi, mu
    return e


def make_phantom(spec):
    rng = np.random.default_rng(1000003 * spec.seed + 7)
    out = []
    if spec.phantom == "head":
        # Head-like layout: a dense shell, a water-like interior and a few low
        # contrast features; positions and sizes jittered by the seed.
        s = spec.fov / 250.0
        j = lambda a: a * (1.0 + 0.05 * rng.uniform(-1, 1))
        d = lambda: 2.0 * s * rng.uniform(-1, 1)
        out.append(_E(0, 0, 0, j(92 * s), j(115 * s), 100.0, 0.0, 2.0 * MU_WATER))
        out.append(_E(0, -2 * s, 0, j(86 * s), j(108 * s), 95.0, 0.0, -1.0 * MU_WATER))
        feats = [(-24, 12, 0, 12, 30, 25, -0.32, -0.05), (24, 12, 0, 16, 40, 25, 0.32, -0.05),
                 (0, 38, -4, 20, 24, 20, 0.0, 0.03), (0, 8, 5, 5, 5, 5, 0.0, 0.04), (0, -12, 0, 5, 2.5, 3, 0.0, 0.04),
                 (-9, -62, 0, 5, 2.5, 3, 0.0, 0.03), (0, -62, 0, 2.5, 2.5, 3, 0.0, 0.03),
                 (7, -62, 0, 2.5, 5, 3, 0.0, 0.03)]
        for (cx, cy, cz, ax, ay, az, phi, c) in feats:
            out.append(_E(cx * s + d(), cy * s + d(), cz, j(ax * s), j(ay * s), az, phi, c * MU_WATER))
    elif spec.phantom == "water_random":
        out.append(_E(0, 0, 0, 160.0, 120.0, 1.0e4, 0.0, MU_WATER))
        zr = 0.5 * spec.V * spec.feed / spec.P
        for _ in range(spec.n_random):
            while True:
                cx, cy = rng.uniform(-140, 140), rng.uniform(-100, 100)
                if (cx / 140.0) ** 2 + (cy / 100.0) ** 2 < 1.0:
                    break
            hu = rng.uniform(-1000, 1500)
            out.append(_E(cx, cy, rng.uniform(-zr, zr), rng.uniform(5, 35), rng.uniform(5, 35), rng.uniform(5, 50),
                          rng.uniform(0, math.pi), MU_WATER * hu / 1000.0))
    elif spec.phantom == "body_random":
        out.append(_E(0, 0, 0, 200.0, 150.0, 1.0e4, 0.0, MU_WATER))
        zr = 0.5 * spec.V * spec.feed / spec.P
        for _ in range(spec.n_random):
            while True:
                cx, cy = rng.uniform(-180, 180), rng.uniform(-130, 130)
                if (cx / 180.0) ** 2 + (cy / 130.0) ** 2 < 1.0:
                    break
            hu = rng.uniform(-1000, 1500)
            out.append(_E(cx, cy, rng.uniform(-zr, zr), rng.uniform(4, 30), rng.uniform(4, 30), rng.uniform(4, 40),
                          rng.uniform(0, math.pi), MU_WATER * hu / 1000.0))
    elif spec.phantom == "fov_random":
        # elliptical water body filling 80 % of the FOV, seeded inserts inside
        a, b = 0.4 * spec.fov, 0.3 * spec.fov
        out.append(_E(0, 0, 0, a, b, 1.0e4, 0.0, MU_WATER))
        zr = 0.5 * spec.V * spec.feed / spec.P
        r = 0.08 * spec.fov
        for _ in range(spec.n_random):
            while True:
                cx, cy = rng.uniform(-0.85 * a, 0.85 * a), rng.uniform(-0.85 * b, 0.85 * b)
                if (cx / (0.85 * a)) ** 2 + (cy / (0.85 * b)) ** 2 < 1.0:
                    break
            hu = rng.uniform(-1000, 1500)
            out.append(_E(cx, cy, rng.uniform(-zr, zr), rng.uniform(0.2, 1) * r, rng.uniform(0.2, 1) * r,
                          rng.uniform(0.2, 1.5) * r, rng.uniform(0, math.pi), MU_WATER * hu / 1000.0))
    else:
        raise ValueError(spec.phantom)
    return out


def small(seed=0):
    return ScanSpec("small", sid=595.0, sdd=1085.6, nch=672, dbeta=0.0012, c0=336.25, nr=16, row_iso=0.6, P=1160,
                    rotations=3, feed=9.6, i0=1e5, nx=256, ny=256, fov=250.0, slice_thickness=1.0, slice_pitch=1.0,
                    n_slices=16, window=T.FILTER_REFERENCE, phantom="head", seed=seed)


def rows64(seed=0):
    dbeta = 2.0 * math.asin(250.0 / 541.0) / 887.0
    return ScanSpec("rows64", sid=541.0, sdd=949.0, nch=888, dbeta=dbeta, c0=443.75, nr=64, row_iso=0.625, P=984,
                    rotations=10, feed=39.37, i0=2e5, nx=512, ny=512, fov=360.0, slice_thickness=1.0,
                    slice_pitch=1.0, n_slices=300, window=T.FILTER_SHEPP_LOGAN, phantom="water_random", seed=seed,
                    n_random=20)


def rows64_short(seed=0):
    """The rows64 scanner over 2.5 rotations and 60 slices: a profiling-size
    case of the same kernels (about 1.5 GB on the device)."""
    spec = rows64(seed=seed)
    spec.name = "rows64_short"
    spec.rotations = 2.5
    spec.n_slices = 60
    return spec


def ffs(seed=0):
    """Flying focal spot in phi and z: 736 ch x 32 rows (0.6 mm), 2304 readings
    per rotation (1152 views/rotation x 2 focal positions) cycling through
    the 4 focal states, 8 rotations, pitch 0.8; 1472 effective channels x 64
    effective rows, 576 views/rotation after merging. 40 seeded ellipsoids,
    I0 1.5e5, 512^2 x 200 slices 0.75 mm thick at a 0.5 mm pitch (200 x 0.75 mm
    would exceed the 123 mm scanned), 500 mm FOV."""
    return ScanSpec("ffs", sid=595.0, sdd=1085.6, nch=736, dbeta=0.0011844, c0=366.25, nr=32, row_iso=0.6,
                    P=2304, rotations=8, feed=0.8 * 32 * 0.6, i0=1.5e5, nx=512, ny=512, fov=500.0,
                    slice_thickness=0.75, slice_pitch=0.5, n_slices=200, window=T.FILTER_REFERENCE,
                    phantom="body_random", seed=seed, n_random=40, ffs_mode=T.FFS_PHIZ)


def batch_specs(seed=0, n=24, reduced=False):
    """Uneven helical scans with seeded shapes: rows in {16, 32, 64} (0.6 mm),
    672-888 channels, 984-1160 views/rotation, 2-12 rotations, pitch 0.5-1.5,
    200-500 mm FOV, 256^2 or 512^2 matrix, 0.75-1.5 mm slices, I0 5e4-3e5, an
    elliptical body with seeded inserts. The scanner is the small one's (SID
    595, SDD 1085.6) with the fan spacing set for a 520 mm acquisition FOV.
    Slices cover the scan's central (rotations - 1.5) turns of table feed.
    reduced=True shrinks every scan (channels / 4, rows / 4, views / 8, at
    most 3 rotations, 64^2 matrix, at most 4 slices) for tests."""
    rng = np.random.default_rng(7919 * seed + 17)
    out = []
    for i in range(n):
        rows = int(rng.choice([16, 32, 64]))
        nch = int(rng.integers(672, 889))
        P = int(rng.integers(984, 1161))
        rot = int(rng.integers(2, 13))
        pitch = float(rng.uniform(0.5, 1.5))
        fov = float(rng.uniform(200.0, 500.0))
        mat = int(rng.choice([256, 512]))
        thick = float(rng.uniform(0.75, 1.5))
        i0 = float(rng.uniform(5e4, 3e5))
        if reduced:
            rows, nch, P, rot, mat = max(4, rows // 4), nch // 4, P // 8, min(rot, 3), 64
        row_iso = 0.6 if not reduced else 2.4
        feed = pitch * rows * row_iso
        n_slices = max(2, int((rot - 1.5) * feed / thick))
        if reduced:
            n_slices = min(n_slices, 4)
        dbeta = 2.0 * math.asin(260.0 / 595.0) / (nch - 1)
        out.append(ScanSpec("batch%d" % i, sid=595.0, sdd=1085.6, nch=nch, dbeta=dbeta, c0=0.5 * (nch - 1) + 0.25,
                            nr=rows, row_iso=row_iso, P=P, rotations=rot, feed=feed, i0=i0, nx=mat, ny=mat, fov=fov,
                            slice_thickness=thick, slice_pitch=thick, n_slices=n_slices, window=T.FILTER_REFERENCE,
                            phantom="fov_random", seed=1000 * seed + i, n_random=12))
    return out


def tiny_ffs(seed=0, mode=T.FFS_PHIZ, nch=64, nr=4, P=128, rotations=3, nx=32, n_slices=4):
    """Reduced flying-focal-spot scan for tests."""
    spec = tiny(seed=seed, nch=nch, nr=nr, P=P, rotations=rotations, nx=nx, n_slices=n_slices)
    spec.name = "tiny_ffs"
    spec.ffs_mode = mode
    return spec


def tiny(seed=0, nch=96, nr=8, P=96, rotations=3, nx=32, n_slices=4, window=T.FILTER_REFERENCE):
    """Reduced scan for CPU tests: the small scanner with a coarser detector."""
    scale = 672.0 / nch
    return ScanSpec("tiny", sid=595.0, sdd=1085.6, nch=nch, dbeta=0.0012 * scale, c0=nch / 2 + 0.25, nr=nr,
                    row_iso=0.6 * 16.0 / nr, P=P, rotations=rotations, feed=9.6, i0=1e5, nx=nx, ny=nx, fov=250.0,
                    slice_thickness=1.0, slice_pitch=1.0, n_slices=n_slices, window=window, phantom="head",
                    seed=seed)


WORKLOADS = {"small": small, "rows64": rows64, "rows64_short": rows64_short, "ffs": ffs, "tiny": tiny}
