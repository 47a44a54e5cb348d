"""Extracts the halo/pole exchange tables of the reference's communication
self-test into a compact JSON fixture.

Source: kernels/NICAM/communication/reference/msg.pe00000{0,1}.Ubuntu-gnu-ompi
of IcoAtmosBenchmark_v1 (gl4, rl0, vlayer 20, 2 MPI ranks; printed by
COMM_debugtest, communication/src/mod_comm.f90:2120-2481).  Each rank's log
holds, for the phases "TEST start" (initial labels), "Communication start"
(after COMM_data_transfer) and "pole fill start" (after COMM_var), the
(prc,rgnid) and (i,j) labels of every point at k = kmin, for its 5 regions
(18x18 tables, rows printed j = 18..1) and the 2 pole regions (6 points).
Values are printed with Fortran I3; "***" marks a value that does not fit
(only the -999 fill of untouched halo points).  In the JSON, that is null.

Run once, where the reference is mounted:
    python tests/golden/make_comm_golden.py /path/to/IcoAtmosBenchmark_v1
"""
import json
import re
import sys
from pathlib import Path

PAIR = re.compile(r"\((.{3}),(.{3})\)")
ROW = re.compile(r"^\s*(-?\d+)\|(.*)$")
PHASES = [("init", "+++ TEST start"), ("comm", "+++ Communication start"), ("polefill", "+++ pole fill start")]


def _val(s):
    s = s.strip()
    return None if s.startswith("*") else int(s)


def parse(path: Path, gall_1d: int = 18, lall: int = 5):
    lines = path.read_text().splitlines()
    starts = []
    for key, marker in PHASES:
        starts.append(next(n for n, ln in enumerate(lines) if ln.strip() == marker))
    starts.append(len(lines))
    out = {}
    for (key, _), a, b in zip(PHASES, starts[:-1], starts[1:]):
        block = lines[a:b]
        res = {}
        for tag, head in (("prc_rgn", "##### (prc,rgnid) #####"), ("ij", "##### (i,j) #####")):
            h = next(n for n, ln in enumerate(block) if ln.strip() == head)
            rows = []
            for ln in block[h + 1:]:
                if ln.strip().startswith("#####") or ln.strip().startswith("+++"):
                    break
                m = ROW.match(ln)
                if m and "(" in m.group(2):
                    rows.append([[_val(x), _val(y)] for x, y in PAIR.findall(m.group(2))])
            regions = [rows[r * gall_1d:(r + 1) * gall_1d][::-1] for r in range(lall)]  # index [l][j-1][i-1]
            poles = rows[lall * gall_1d:lall * gall_1d + 2]
            assert all(len(r) == gall_1d for g in regions for r in g), path
            assert len(poles) == 2 and all(len(p) == 6 for p in poles), path
            res[tag] = regions
            res["pole_" + tag] = poles
        out[key] = res
    return out


def main(ref_root: str):
    base = Path(ref_root) / "kernels/NICAM/communication/reference"
    fixture = {
        "source": "kernels/NICAM/communication/reference/msg.pe00000{0,1}.Ubuntu-gnu-ompi",
        "glevel": 4, "rlevel": 0, "vlayer": 20, "nprocs": 2, "k": "kmin",
        "ranks": [parse(base / f"msg.pe00000{r}.Ubuntu-gnu-ompi") for r in range(2)],
    }
    # the intel and pgi logs must hold the same tables
    for comp in ("intel", "pgi"):
        for r in range(2):
            assert parse(base / f"msg.pe00000{r}.Ubuntu-{comp}-ompi") == fixture["ranks"][r], (comp, r)
    dst = Path(__file__).with_name("comm_gl04rl00_2rank.json")
    dst.write_text(json.dumps(fixture, separators=(",", ":")))
    print(dst, dst.stat().st_size, "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_comm_golden.py <root of the IcoAtmosBenchmark_v1 checkout>")
    main(sys.argv[1])
