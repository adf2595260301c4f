"""TEST ORACLE — CPU restatement of the device DAG build's walk (engine csrc/dag.cu).

Test infrastructure only (tests/ import it; the product never does).  The host build
(Program::build_dag) keeps, per storage object, a list of the accesses not yet covered by a
later write and scans it newest first; the device build keeps no lists: every access walks all
earlier accesses of its object newest first and decides from what it met on the way.  This
module runs that walk on the CPU over a program's regions (pp_hmatrix_program_regions), so a
test can check, without a GPU, that the walk's rule yields exactly the host's typed edges:

  * accesses of the same instruction are skipped;
  * an access that does not overlap this region is skipped;
  * an access covered by a write met earlier in the walk is skipped (the host dropped it when
    that write was inserted);
  * otherwise the pair gets flow (write then read, 1), anti (read then write, 2) or out (write
    then write, 4); a write covering this region ends the walk.

The dependency types are those of the reference's rts/dependency.h:9-18; the overlap and cover
tests are on (first row, first column, rows, columns) rectangles of one object.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np


def _overlap(a, b):
    return a[0] < b[0] + b[2] and b[0] < a[0] + a[2] and a[1] < b[1] + b[3] and b[1] < a[1] + a[3]


def _covers(a, b):
    return a[0] <= b[0] and b[0] + b[2] <= a[0] + a[2] and a[1] <= b[1] and b[1] + b[3] <= a[1] + a[3]


def walk_edges(regions):
    """regions: int rows (task, object, row0, col0, rows, cols, read_only) in program order.
    Returns {(pred, task): type bits} as the device walk builds it."""
    by_obj = defaultdict(list)
    for k, (t, o, r0, c0, nr, nc, ro) in enumerate(np.asarray(regions).tolist()):
        by_obj[o].append((t, (r0, c0, nr, nc), bool(ro)))
    edges = {}
    for acc in by_obj.values():
        for p, (t, rect, ro) in enumerate(acc):
            met = []  # writes met on the way that did not end it
            for q in range(p - 1, -1, -1):
                te, re, roe = acc[q]
                if te == t or not _overlap(re, rect):
                    continue
                if any(_covers(w, re) for w in met):
                    continue
                d = 1 if (not roe and ro) else 2 if (roe and not ro) else 4 if (not roe and not ro) else 0
                if d:
                    edges[(te, t)] = edges.get((te, t), 0) | d
                if not roe:
                    if _covers(re, rect):
                        break
                    met.append(re)
    return edges
