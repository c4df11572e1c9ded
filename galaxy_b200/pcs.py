"""The reference's particle files (.pcs) and the pcs2dmp-style start of a run.

A .pcs file is a Fortran unformatted sequential file (4-byte record length
before and after every record), as SRC/lib15/loadup.f:36-140 reads it:

    record 0   nsp(3) int32, mcoor int32, l int32, t real32, pm real32,
               log (logical, int32): populations, coordinates per particle,
               particles per record, time, particle mass, perturber present
    record 1   (only when log) the perturber: xptrb(3), vptrb(3), mptbr, eptbr
    then       records of min(l, remaining) * mcoor real32 values: the
               particles one after another, x(ndim), v(ndim) [, mass when
               mcoor is odd], in the model's units

loadup converts positions to grid units with x * lscale, velocities with
v / gvfac, gvfac = 1 / (lscale ts) (SRC/lib15/setrun.f:872-873), and the
particle mass with pm lscale^3 ts^2 (loadup.f:97-99); particles at the exact
origin are discarded (loadup.f:193-199).
"""
import struct

import numpy as np


class Pcs:
    """Contents of a .pcs file (records in the model's units)."""

    def __init__(self, nsp, mcoor, per_record, t, pm, records, perturber=None):
        self.nsp = tuple(int(v) for v in nsp)
        self.mcoor = int(mcoor)
        self.per_record = int(per_record)
        self.t = float(t)
        self.pm = float(pm)
        self.records = np.ascontiguousarray(records, np.float32).reshape(-1, self.mcoor)
        self.perturber = perturber

    @property
    def n(self):
        return self.records.shape[0]

    @property
    def ndim(self):
        return (self.mcoor - (self.mcoor % 2)) // 2

    def grid_units(self, lscale, ts):
        """(records (n, 2 ndim) float32 in grid units, particle mass in
        internal units) as loadup stores them; particles at the origin
        dropped."""
        nd = self.ndim
        r = self.records.astype(np.float64)
        keep = np.any(r[:, :nd] != 0.0, axis=1)
        out = np.empty((int(keep.sum()), 2 * nd), np.float32)
        out[:, :nd] = (r[keep, :nd] * lscale).astype(np.float32)
        out[:, nd:] = (r[keep, nd:2 * nd] * (lscale * ts)).astype(np.float32)
        pmass = self.pm * lscale ** 3 * ts ** 2
        return out, pmass


def _records(buf):
    off = 0
    while off < len(buf):
        (n,) = struct.unpack_from("<i", buf, off)
        body = buf[off + 4:off + 4 + n]
        (n2,) = struct.unpack_from("<i", buf, off + 4 + n)
        if n2 != n:
            raise ValueError("corrupt .pcs record markers")
        yield body
        off += 8 + n


def read_pcs(path):
    buf = open(path, "rb").read()
    it = _records(buf)
    head = next(it)
    nsp0, nsp1, nsp2, mcoor, l, t, pm, log = struct.unpack_from("<5iffi", head)
    pert = None
    if log:
        pert = np.frombuffer(next(it), np.float32).copy()
    nbod = nsp0 + nsp1 + nsp2
    vals = [np.frombuffer(b, np.float32) for b in it]
    rec = np.concatenate(vals) if vals else np.zeros(0, np.float32)
    if rec.size != nbod * mcoor:
        raise ValueError(f".pcs holds {rec.size} values, header says {nbod} x {mcoor}")
    return Pcs((nsp0, nsp1, nsp2), mcoor, l, t, pm, rec, pert)


def write_pcs(path, pcs):
    """The same layout: header, optional perturber, records of per_record particles."""
    def rec(b):
        return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))
    out = [rec(struct.pack("<5iffi", *pcs.nsp, pcs.mcoor, pcs.per_record, pcs.t, pcs.pm,
                           1 if pcs.perturber is not None else 0))]
    if pcs.perturber is not None:
        out.append(rec(np.ascontiguousarray(pcs.perturber, np.float32).tobytes()))
    r = pcs.records
    for s in range(0, r.shape[0], pcs.per_record):
        out.append(rec(np.ascontiguousarray(r[s:s + pcs.per_record], np.float32).tobytes()))
    open(path, "wb").write(b"".join(out))


def start_run(cfg, pcs, lscale, ts, tcent=True):
    """pcs2dmp's set-up of a run (SRC/progs/pcs2dmp.f:56-104): the grid and
    Green table, the particles in grid units, their mass, the field and the
    half-step velocity offset of time centring (tmcent.f:83-90).  Returns a
    Galaxy ready for step()."""
    from . import Galaxy
    rec, pmass = pcs.grid_units(lscale, ts)
    cfg.pmass = pmass
    gal = Galaxy(cfg)
    gal.greenm()
    gal.loadup(rec)
    gal.masset()
    if tcent:
        gal.findf(False)
        gal.tmcent(True)
    return gal
