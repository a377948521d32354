"""Programmatic dependent launch guard (static, CPU).

On small 2D grids the step graph launches its kernels with programmatic stream
serialisation (solver.cu, launch_k with s->pdl). Such a kernel may start
before its predecessor has finished. It must therefore wait
(griddepcontrol.wait, pdl_enter()) before touching memory: every kernel
launched through launch_k(s->pdl, ...) must begin with pdl_enter().
"""
import glob
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "simplevofsolver_b200", "csrc")


def pdl_launched_kernels():
    text = open(os.path.join(CSRC, "solver.cu")).read()
    return sorted(set(re.findall(r"launch_k\(\s*s->pdl\s*,\s*(\w+)\s*,", text)))


def first_statement(kernel):
    for path in glob.glob(os.path.join(CSRC, "*.cu")):
        text = open(path).read()
        m = re.search(r"__global__\s+void[^;{]*?\b" + kernel + r"\s*\(", text)
        if not m:
            continue
        body = text[text.index("{", m.end()) + 1:]
        body = re.sub(r"//[^\n]*", "", body)
        return body.strip().split(";", 1)[0].strip()
    raise AssertionError(f"definition of {kernel} not found")


def test_pdl_launches_exist():
    names = pdl_launched_kernels()
    assert {"k_geom", "k_predict", "k_project", "k_cfl"} <= set(names), names


def test_every_pdl_kernel_waits_first():
    for k in pdl_launched_kernels():
        assert first_statement(k) == "pdl_enter()", (k, first_statement(k))
