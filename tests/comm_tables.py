"""Helpers to reproduce the reference communication self-test tables
(COMM_debugtest, communication/src/mod_comm.f90:2120-2481) with the oracle's
emulated ranks or with a single-process halo plan, in the fixture format of
tests/golden/make_comm_golden.py."""
import numpy as np


def i3(x):
    """Fortran I3 of int(x): values that do not fit print as ***, stored as None."""
    v = int(x)
    return v if -99 <= v <= 999 else None


def debugtest_init(nprocs, lall, gall_1d, kall, kmin, kmax, rgnid_of, have_sgp_of):
    """Initial labels of COMM_debugtest (:2153-2192) for every rank."""
    gall = gall_1d * gall_1d
    gmin, gmax = 2, gall_1d - 1
    var, var_pl = [], []
    for p in range(1, nprocs + 1):
        v = np.full((4, lall, kall, gall), -999.0)
        vp = np.full((4, 2, kall, 6), -999.0)
        for l in range(1, lall + 1):
            rg = rgnid_of(p, l)
            for j in range(gmin, gmax + 1):
                for i in range(gmin, gmax + 1):
                    ij = gall_1d * (j - 1) + i - 1
                    v[0, l - 1, kmin - 1:kmax, ij] = p
                    v[1, l - 1, kmin - 1:kmax, ij] = rg
                    v[2, l - 1, kmin - 1:kmax, ij] = i
                    v[3, l - 1, kmin - 1:kmax, ij] = j
            if have_sgp_of(p, l):
                v[:, l - 1, kmin - 1:kmax, 0] = -1.0
        for l in range(1, 3):
            for ij in range(1, 7):
                vp[0, l - 1, kmin - 1:kmax, ij - 1] = -p
                vp[1, l - 1, kmin - 1:kmax, ij - 1] = -l
                vp[2, l - 1, kmin - 1:kmax, ij - 1] = -ij
                vp[3, l - 1, kmin - 1:kmax, ij - 1] = -ij
        var.append(v)
        var_pl.append(vp)
    return var, var_pl


def set_pole_halo_labels(var, nprocs, lall, gall_1d, kmin, kmax, rgnid_of, vert_num):
    """The relabelling before COMM_var (:2363-2393)."""
    gmin, gmax = 2, gall_1d - 1
    for p in range(1, nprocs + 1):
        for l in range(1, lall + 1):
            rg = rgnid_of(p, l)
            for corner, (i, j) in ((1, (gmin, gmax + 1)), (3, (gmax + 1, gmin))):  # N, S
                if vert_num[rg - 1, corner] == 5:
                    ij = gall_1d * (j - 1) + i - 1
                    var[p - 1][:, l - 1, kmin - 1:kmax, ij] = np.array([p, rg, i, j], float)[:, None]


def tables(v, vp, kmin, gall_1d, lall):
    """Fixture-format tables of one rank at k = kmin."""
    k = kmin - 1
    out = {}
    for tag, (a, b) in (("prc_rgn", (0, 1)), ("ij", (2, 3))):
        regs = []
        for l in range(lall):
            g = []
            for j in range(gall_1d):
                g.append([[i3(v[a, l, k, j * gall_1d + i]), i3(v[b, l, k, j * gall_1d + i])] for i in range(gall_1d)])
            regs.append(g)
        out[tag] = regs
        out["pole_" + tag] = [[[i3(vp[a, l, k, n]), i3(vp[b, l, k, n])] for n in range(6)] for l in range(2)]
    return out
