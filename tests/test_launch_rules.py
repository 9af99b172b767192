"""Source rules that make programmatic dependent launch safe.

Every kernel is launched through ``qgn::launch`` (csrc/launch.cuh), which lets the next grid in
the stream start before the current one has finished.  That is only correct if every kernel
waits for its prerequisite grids before it touches memory, so the first statement of every
``__global__`` body must be ``QGN_PDL_ENTRY();`` and no ``<<<...>>>`` launch may bypass the
launcher.
"""
import os
import re

import pytest

CSRC = os.path.join(os.path.dirname(__file__), "..", "qgn_fortran_b200", "csrc")


def sources():
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh")):
            with open(os.path.join(CSRC, f)) as fh:
                yield f, fh.read()


def strip_comments(s):
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def kernel_bodies(s):
    """(name, text after the opening brace) of every __global__ definition."""
    for m in re.finditer(r"__global__", s):
        brace = s.find("{", m.end())
        semi = s.find(";", m.end())
        if semi != -1 and semi < brace:
            continue   # a declaration
        head = s[m.end():brace]
        name = re.findall(r"(\w+)\s*\(", head)
        yield (name[-1] if name else "?"), s[brace + 1:]


def test_every_kernel_waits_for_its_prerequisites():
    n = 0
    for f, s in sources():
        s = strip_comments(s)
        for name, body in kernel_bodies(s):
            n += 1
            first = body.lstrip().split(";", 1)[0].strip()
            assert first == "QGN_PDL_ENTRY()", f"{f}: kernel {name} does not start with QGN_PDL_ENTRY()"
    assert n >= 50


@pytest.mark.parametrize("f", [f for f, _ in sources()])
def test_no_triple_chevron_launch(f):
    s = dict(sources())[f]
    assert "<<<" not in strip_comments(s), f"{f} launches a kernel without qgn::launch"
