"""The work split of the L2-staged small-level cycle (CPU): csrc/ssa_small_plan.h's chunks
and staged row windows, compiled here with g++, for the down steps of the level chains
mg_plan builds on many grid shapes, with the cluster's 8 CTAs and for the single-CTA steps."""
import os
import shutil
import subprocess

import pytest

from tests.test_small_plan import mg_chain

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path_factory.mktemp("split") / "small_split_check")
    subprocess.run([gxx, "-O1", "-std=c++17", "-I", os.path.join(REPO, "pismv0.7.3_b200", "csrc"),
                    os.path.join(REPO, "tests", "small_split_check.cc"), "-o", exe], check=True)
    return exe


SHAPES = [(801, 801), (401, 401), (1601, 1601), (201, 131), (130, 97), (45, 44), (64, 64), (5, 201), (201, 5),
          (33, 17), (7, 7), (9, 300), (1000, 3), (61, 121)]


@pytest.mark.parametrize("cta_cells", [4096, 16384])
@pytest.mark.parametrize("shape", SHAPES)
def test_chunks_cover_items_and_windows_hold_their_rows(checker, shape, cta_cells):
    lev, first = mg_chain(*shape, cta_cells=cta_cells)
    if lev is None:
        pytest.skip("no hierarchy")
    lines = []
    for l in range(first, len(lev) - 1):
        Mx, My, ax, ay = lev[l]
        Mxc, Myc = lev[l + 1][0], lev[l + 1][1]
        for parts, local in ((8, 1024), (1, 1 << 30)):
            lines.append(f"{Mx} {My} {ax} {ay} {Mxc} {Myc} {parts} {local}")
    out = subprocess.run([checker], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    res = out.stdout.split("\n")[:len(lines)]
    assert all(r.startswith("ok") for r in res), list(zip(lines, res))
