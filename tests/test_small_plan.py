"""The split of the small multigrid levels over the cluster's CTAs (CPU): the plan of
csrc/ssa_small_plan.h, compiled here with g++, for the level chains mg_plan builds on many
grid shapes.  Every level's blocks must cover its cells once, nest (the fine cells of a
coarse cell's aggregate on the coarse cell's CTA), fit the per-CTA arrays the kernel indexes,
and the owner lookup must find each row's and column's block."""
import json
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAX_SMEM = 220 * 1024
CTAS = 8


def mg_chain(Mx, My, coarse_dim=4, cta_cells=4096, max_levels=16):
    """mg_plan (csrc/ssa_mg.cu): the coarse levels (Mx, My, ax, ay) and the first small one"""
    if Mx <= coarse_dim and My <= coarse_dim:
        return None, None
    fax, fay = (2 if Mx > coarse_dim else 1), (2 if My > coarse_dim else 1)
    mx, my = (Mx + fax - 1) // fax, (My + fay - 1) // fay
    lev = []
    while len(lev) < max_levels:
        if mx <= coarse_dim and my <= coarse_dim:
            lev.append([mx, my, 1, 1])
            break
        ax, ay = (2 if mx > coarse_dim else 1), (2 if my > coarse_dim else 1)
        lev.append([mx, my, ax, ay])
        mx, my = (mx + ax - 1) // ax, (my + ay - 1) // ay
    if lev[-1][0] > coarse_dim or lev[-1][1] > coarse_dim:
        return None, None
    first = len(lev) - 1
    while first > 0 and lev[first - 1][0] * lev[first - 1][1] <= cta_cells:
        first -= 1
    return lev, first


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path_factory.mktemp("sp") / "check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(REPO, "pismv0.7.3_b200", "csrc"),
                    os.path.join(REPO, "tests", "small_plan_check.cc"), "-o", exe], check=True)
    return exe


SHAPES = [(801, 801), (401, 401), (1601, 1601), (201, 201), (41, 41), (45, 44), (64, 64), (33, 33), (17, 17),
          (9, 9), (5, 201), (5, 61), (201, 3), (401, 3), (23, 19), (2047, 2049), (3, 5000), (5000, 3), (7, 7),
          (100, 37), (6, 6)]


def test_plans_cover_nest_and_fit(driver):
    chains = []
    for Mx, My in SHAPES:
        lev, first = mg_chain(Mx, My)
        if lev is None:
            continue
        small = lev[first:]
        chains.append((Mx, My, small))
    lines = ["%d %d %s" % (len(s), MAX_SMEM, " ".join("%d %d %d %d" % tuple(l) for l in s)) for _, _, s in chains]
    out = subprocess.run([driver], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    plans = [json.loads(l) for l in out.stdout.splitlines()]
    assert len(plans) == len(chains)
    fitted = 0
    for (Mx, My, small), P in zip(chains, plans):
        if not P["ok"]:
            continue
        fitted += 1
        Pr, Pc = P["Pr"], P["Pc"]
        assert 1 <= Pr * Pc <= CTAS and P["smem"] <= MAX_SMEM
        end = 0
        for l, (mx, my, ax, ay) in enumerate(small):
            L = P["levels"][l]
            rb, cb, mi, mj = L["rb"], L["cb"], L["mi"], L["mj"]
            # the blocks cover the level once, none empty
            assert rb[0] == 0 and rb[-1] == mx and cb[0] == 0 and cb[-1] == my
            assert all(rb[p] < rb[p + 1] for p in range(Pr)) and all(cb[q] < cb[q + 1] for q in range(Pc))
            assert mi == max(rb[p + 1] - rb[p] for p in range(Pr)) and mj == max(cb[q + 1] - cb[q] for q in range(Pc))
            # the owner lookup
            assert L["row_owner"] == [next(p for p in range(Pr) if rb[p] <= i < rb[p + 1]) for i in range(mx)]
            assert L["col_owner"] == [next(q for q in range(Pc) if cb[q] <= j < cb[q + 1]) for j in range(my)]
            # the arrays: 10 float4 and 2 float2 per slot, then two padded float2 arrays with a
            # halo ring, levels one after another
            assert L["off4"] >= end and L["off4"] % 128 == 0
            assert L["off2"] == L["off4"] + 160 * mi * mj
            assert L["offp"] == L["off2"] + 16 * mi * mj
            end = L["offp"] + 16 * (mi + 2) * (mj + 2)
            assert end <= P["smem"]
            # nesting: a coarse cell's aggregate lives on its CTA
            if l + 1 < len(small):
                C = P["levels"][l + 1]
                for I in range(small[l + 1][0]):
                    for i in range(I * ax, min(I * ax + ax, mx)):
                        assert L["row_owner"][i] == C["row_owner"][I], (Mx, My, l, I, i)
                for J in range(small[l + 1][1]):
                    for j in range(J * ay, min(J * ay + ay, my)):
                        assert L["col_owner"][j] == C["col_owner"][J], (Mx, My, l, J, j)
    # the benchmark grid and the ensemble grid use the shared-memory cycle
    ok = {(Mx, My): P["ok"] for (Mx, My, _), P in zip(chains, plans)}
    assert ok[(801, 801)] and ok[(401, 401)] and ok[(1601, 1601)]
    assert fitted >= len(chains) - 3


def test_plan_rejects_too_much_shared_memory(driver):
    lev, first = mg_chain(801, 801)
    small = lev[first:]
    line = "%d %d %s" % (len(small), 4096, " ".join("%d %d %d %d" % tuple(l) for l in small))
    out = subprocess.run([driver], input=line + "\n", capture_output=True, text=True, check=True)
    assert json.loads(out.stdout) == {"ok": False}
