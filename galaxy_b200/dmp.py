"""The reference's restart dumps (.dmp) of polar-grid runs.

dumpp (SRC/lib15/dumpp.f:40-230) writes a Fortran unformatted sequential
file (4-byte record length before and after every record):

    hedrec          hedrc1: cvers, ngrid, .., lscale, ts, nlists, ng, nbod,
                    ncmp, pmass, softl, .., nsect, jmass, .., tsoft, ndimen
                    (SRC/lib15/hedrec.f, hedrc1); hedrcg per grid: nr, na,
                    ng, rgrid, gamma, uoffs, ngz, dzg, s3lmax, lg(1..ng);
                    hedrcc per population
    run record      irun, istep, noff, ncen(4), nshort, nrsup, suppl, n, ...
    (supplementary forces, perturber, centroid records when present)
    list record     numprocs, myid, particles on this node, nwpp, the head
                    of every linked list (word offsets, -1 = empty)
    random state
    grdmss(:, 1)    the solve's mass array (scaled)
    per zone >= 2   lstep(1), grdmoz(:, zone); lstep(2), grdmss(:, zone)
    particles       nwpp words each: coordinates (x, v), flags, and the word
                    offset of the next particle of its list
    (off-grid index list)

The lists are the time-step zones: list i < nlists holds zone i (no guard
zones), list nlists the particles off the grid.  Velocities are in units
of each zone's own step (adjvls.f) and time-centred (the dump requires
tcent).  Single-process dumps of one polar grid (p2d, p3d) are read.
"""
import struct

import numpy as np


def _records(buf):
    off = 0
    while off < len(buf):
        (n,) = struct.unpack_from("<i", buf, off)
        (n2,) = struct.unpack_from("<i", buf, off + 4 + n)
        if n2 != n:
            raise ValueError("corrupt .dmp record markers")
        yield buf[off + 4:off + 4 + n]
        off += 8 + n


class Dmp:
    """Contents of a .dmp file.  records: (n, 2 ndim) float32 in grid units
    with velocities in zone-step units, in the file's particle order; zone:
    1..nzones, nzones + 1 off the grid; mass: the solve's mass array;
    zone_mass[z] = (lstep_old, old array, lstep_new, new array) for z >= 2."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def base_records(self, nstep):
        """records with velocities in base-step units (adjvls(.false.)):
        divided by nstep[zone - 1] for particles on the grid"""
        r = self.records.copy()
        nd = self.ndim
        on = self.zone <= self.nzones
        fac = np.asarray(nstep, np.float32)[np.minimum(self.zone, self.nzones) - 1]
        r[on, nd:] = r[on, nd:] * (np.float32(1) / fac[on])[:, None]
        return r


def read_dmp(path):
    recs = list(_records(open(path, "rb").read()))
    h = recs[0]
    hi = np.frombuffer(h, np.int32)
    hf = np.frombuffer(h, np.float32)
    ngrid, nlists, ng, nbod, ncmp = int(hi[1]), int(hi[7]), int(hi[8]), int(hi[9]), int(hi[10])
    if ngrid != 1:
        raise ValueError("only dumps of a single grid are read")
    lscale, ts, pmass, softl = float(hf[5]), float(hf[6]), float(hf[11]), float(hf[12])
    nsect, tsoft, ndim = int(hi[14]), int(hi[20]), int(hi[21])
    g = recs[1]
    gi = np.frombuffer(g, np.int32)
    gf = np.frombuffer(g, np.float32)
    nr, na, ngg = int(gi[0]), int(gi[1]), int(gi[2])
    ngz = max(int(gi[6]), 1)
    grid = dict(nr=nr, na=na, ng=ngg, rgrid=float(gf[3]), gamma=float(gf[4]),
                uoffs=float(gf[5]), ngz=ngz, dzg=float(gf[7]),
                skipped=[m for m in range(ngg) if gi[9 + m] != 0])
    mesh = nr * na * (ngz if ndim == 3 else 1)
    i = 2 + ncmp
    run = np.frombuffer(recs[i], np.int32)
    irun, istep = int(run[0]), int(run[1])
    # the list record: numprocs, myid, count, nwpp, nlists heads
    i += 1
    while len(recs[i]) != 4 * (4 + nlists):
        i += 1
    lr = np.frombuffer(recs[i], np.int32)
    if int(lr[0]) != 1:
        raise ValueError("only single-process dumps are read")
    count, nwpp = int(lr[2]), int(lr[3])
    heads = [int(v) for v in lr[4:]]
    i += 2  # skip the random generator state
    mass = np.frombuffer(recs[i], np.float32).copy()
    if mass.size != mesh:
        raise ValueError("mass record does not match the grid")
    i += 1
    zone_mass = {}
    z = 2
    while len(recs[i]) == 4 + 4 * mesh:
        (lo,) = struct.unpack_from("<i", recs[i], 0)
        (ln,) = struct.unpack_from("<i", recs[i + 1], 0)
        zone_mass[z] = (lo, np.frombuffer(recs[i][4:], np.float32).copy(),
                        ln, np.frombuffer(recs[i + 1][4:], np.float32).copy())
        i += 2
        z += 1
    nzones = len(zone_mass) + 1
    words = count * nwpp
    got = []
    while sum(len(r) for r in got) < 4 * words:
        got.append(recs[i])
        i += 1
    pt = np.frombuffer(b"".join(got)[:4 * words], np.float32).reshape(count, nwpp)
    nxt = pt.view(np.int32)[:, nwpp - 1]
    zone = np.zeros(count, np.int32)
    for li, hd in enumerate(heads):
        j, seen = hd, 0
        while j >= 0:
            p = j // nwpp
            zone[p] = li + 1 if li < nlists - 1 else nzones + 1
            j = int(nxt[p])
            seen += 1
            if seen > count:
                raise ValueError("corrupt particle list")
    return Dmp(path=path, irun=irun, istep=istep, ndim=ndim, nbod=nbod, lscale=lscale, ts=ts,
               pmass=pmass, softl=softl, nsect=nsect, tsoft=tsoft, grid=grid, mesh=mesh,
               nzones=nzones, records=pt[:, :2 * ndim].copy(), zone=zone, mass=mass,
               zone_mass=zone_mass)
