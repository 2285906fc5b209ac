"""Static checks of the generated PTX jump tables (galop_b200/csrc/gen_dispatch.py).

dispatch_gen.cuh must equal the generator's output, and the wide loop's
control flow must be closed: every branch target exists, and the only
fall-through between labelled blocks is the one the loop is built on (an
arm's S, L, F entry points fall into each other; DB falls into the exit).
In particular, the DIV arms' exact paths (V blocks) are entered only by
their arm's uniform branch and jump back into it (W), and the shared SIN/COS
block (R) and its exit (Z) end in jumps, so no path falls into them and
loops.
"""
from __future__ import annotations

import re
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT / "galop_b200" / "csrc"))
import gen_dispatch as G  # noqa: E402

LABEL = re.compile(r"^([A-Za-z_][A-Za-z0-9_]*%=):\s*(.*)$")
BRANCH = re.compile(r"(@!?\w+\s+)?bra(?:\.uni)?\s+([A-Za-z_][A-Za-z0-9_]*%=);")


def loop_blocks(k: int, profile: int):
    """(label or None, statements) per line of the loop's asm block."""
    text = G.wide_loop(k, profile)
    body = text.split('asm volatile("{\\n\\t', 1)[1].split('\\n\\t}"', 1)[0]
    out = []
    for ln in body.split("\\n\\t"):
        m = LABEL.match(ln)
        out.append((m.group(1), m.group(2)) if m else (None, ln))
    return out


def falls_through(stm: str) -> bool:
    parts = [p.strip() for p in stm.strip().split(";") if p.strip()]
    return not parts or not re.match(r"^bra(\.uni)?\s", parts[-1])


def test_header_is_up_to_date():
    assert (ROOT / "galop_b200" / "csrc" / "dispatch_gen.cuh").read_text() == G.render()


@pytest.mark.parametrize("k", G.KS)
@pytest.mark.parametrize("profile", list(G.PROFILES))
def test_wide_loop_control_flow(k, profile):
    bl = loop_blocks(k, profile)
    labels = set()
    for lab, stm in bl:
        if lab:
            labels.add(lab)
        labels.update(m.group(1) for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*%=):", stm))
    targets = set()
    for _, stm in bl:
        targets.update(m.group(2) for m in BRANCH.finditer(stm))
        for m in re.finditer(r"\.branchtargets ([^;]*);", stm):
            targets.update(t.strip() for t in m.group(1).split(","))
    assert targets <= labels, sorted(targets - labels)[:5]

    everything = " ".join(stm for _, stm in bl)
    cold = [i for i, (lab, _) in enumerate(bl) if lab and lab.startswith("V")]
    assert len(cold) == 4                     # DIV x register/constant divisor x two loop copies
    for i in cold:
        lab, stm = bl[i]
        assert not falls_through(bl[i - 1][1]), (bl[i - 1][0], lab)
        assert stm.rstrip().endswith(f"bra.uni W{lab[1:]};"), lab
        assert f"@!funi bra.uni {lab};" in everything, lab
    # SIN/COS: one block (R) shared by both ops and both copies' F arms, and
    # its exit (Z), entered by the uniform slow-path branch; both end in
    # jumps and nothing falls into them
    for lab, entry in (("R_%=", "bra.uni R_%=;"), ("Z_%=", "@tany bra.uni Z_%=;")):
        (i,) = [j for j, (lb, _) in enumerate(bl) if lb == lab]
        assert not falls_through(bl[i - 1][1]), (bl[i - 1][0], lab)
        assert not falls_through(bl[i][1]), lab
        assert entry in everything, lab
    assert everything.count("bra.uni R_%=;") == 2 * len(G.TRIG_OPS)
    # the exit: D%= is the last label and only DB (right before it) falls into it
    assert bl[-1][0] == "D%=" and bl[-2][0] == "DB%="
    for lab, stm in bl[:-2]:
        if lab and lab.startswith(("X", "D")):
            assert not falls_through(stm), lab
