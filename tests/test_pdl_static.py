"""Source check of the programmatic-dependent-launch rule (CPU only).

A kernel launched through ``launch()`` (csrc/internal.h) may start while its
predecessor on the stream is still running; it is only correct if its first
statement is ``pdl_begin()`` (``griddepcontrol.wait`` before any memory
access, and before any early return).  This test reads the CUDA sources and
checks that rule for every kernel launched that way, and that no such kernel
is also launched with the plain ``<<<...>>>`` syntax elsewhere.  Kernels
written as a ``TTG_BODY`` (csrc/group.cuh) count with their body; cooperative
ones (``TTG_COOP_KERNEL``) are launched without the attribute and are exempt.
"""
import pathlib
import re

CSRC = pathlib.Path(__file__).resolve().parents[1] / "tt-toolbox_b200" / "csrc"


def _sources():
    return {p.name: p.read_text() for p in sorted(CSRC.glob("*.cu"))}


def test_every_pdl_launched_kernel_waits_first():
    src = _sources()
    names = set()
    for text in src.values():
        names.update(re.findall(r"\blaunch\(c,\s*([A-Za-z_][A-Za-z_0-9]*)", text))
    assert names, "no launch() call sites found"
    allsrc = "\n".join(src.values())
    # cooperative kernels are launched without the PDL attribute
    coop = set(re.findall(r"TTG_COOP_KERNEL\((\w+)", allsrc))
    bad = []
    for name in sorted(names - coop):
        m = re.search(r"__global__ void[^;{]*?\b%s\s*\([^{]*\{\n(.*)\n" % re.escape(name), allsrc)
        if m is None:  # a TTG_BODY kernel (group.cuh)
            m = re.search(r"TTG_BODY\(%s\)\s*\([^{]*\{\n(.*)\n" % re.escape(name), allsrc)
        first = None if m is None else m.group(1).strip()
        call = re.match(r"(\w+)(?:<[^>]*>)?\(", first or "")
        if call and first != "pdl_begin();":  # a wrapper: the callee must wait first
            d = re.search(r"__device__[^;{]*?\b%s\s*\([^{]*\{\n(.*)\n" % re.escape(call.group(1)),
                          allsrc)
            first = None if d is None else d.group(1).strip()
        if first != "pdl_begin();":
            bad.append((name, first))
    assert not bad, "kernels launched with launch() that do not start with pdl_begin(): %r" % bad


def test_pdl_kernels_have_one_launch_style():
    src = _sources()
    names = set()
    for text in src.values():
        names.update(re.findall(r"\blaunch\(c,\s*([A-Za-z_][A-Za-z_0-9]*)", text))
    mixed = []
    for fname, text in src.items():
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z_0-9]*)(?:<[^<>;]*>)?<<<", text):
            if m.group(1) in names:
                mixed.append((fname, m.group(1)))
    assert not mixed, "kernels launched both ways: %r" % mixed
