"""Every kernel that the library launches with programmatic dependent launch
waits for its predecessor at entry.

With the ProgrammaticStreamSerialization attribute a kernel may start while
the previous kernel of the stream is still running; only
`griddepcontrol.wait` (`pdl_wait()` in csrc/common.cuh) orders its reads
after the predecessor's writes.  A kernel launched through `launch_pdl`
without that wait reads stale fields on some launches and not on others, so
the rule is checked on the sources: each kernel named in a `launch_pdl` call
is defined, and every definition of it calls `pdl_wait()` before anything
else of substance (within the first statements of its body).
"""
import os
import re

CSRC = os.path.join(os.path.dirname(__file__), "..", "chapsim1.0_b200", "csrc")


def _sources():
    out = {}
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cuh")):
            with open(os.path.join(CSRC, name)) as fh:
                out[name] = fh.read()
    return out


def _pdl_kernels(src):
    names = set()
    for text in src.values():
        names.update(re.findall(r"launch_pdl\(\s*[^,()]+,\s*(k_\w+)", text))
        # launch_cluster(pdl, cluster size, kernel, ...): the cluster launches of the plane transforms
        names.update(re.findall(r"launch_cluster\(\s*[^,()]+,\s*[^,()]+,\s*(k_\w+)", text))
    return names


def _bodies(src, kernel):
    pat = re.compile(r"__global__[^;{}]*?\b" + re.escape(kernel) + r"\s*\(")
    for fname, text in src.items():
        for m in pat.finditer(text):
            brace = text.index("{", m.end())
            yield fname, text[brace + 1:brace + 1 + 240]


def test_pdl_kernels_wait_at_entry():
    src = _sources()
    kernels = _pdl_kernels(src)
    assert len(kernels) >= 15, sorted(kernels)  # the step's kernels, the dt rule, the pressure stage
    for k in sorted(kernels):
        bodies = list(_bodies(src, k))
        assert bodies, f"{k}: launched with launch_pdl but no __global__ definition found"
        for fname, head in bodies:
            assert "pdl_wait();" in head, f"{k} ({fname}): no pdl_wait() at entry"


def test_check_rejects_a_kernel_without_the_wait():
    src = {"a.cuh": "template <int S>\n__global__ void __launch_bounds__(256, 2) k_demo(Geo g, double* x) {\n"
                    "    const int i = threadIdx.x;\n    x[i] = 0.0;\n}\n",
           "b.cu": "    CK(launch_pdl(ctx->pdl, k_demo<4>, grid, 256, 0, s, g, x));\n"}
    assert _pdl_kernels(src) == {"k_demo"}
    (fname, head), = list(_bodies(src, "k_demo"))
    assert fname == "a.cuh" and "pdl_wait();" not in head
    src["a.cuh"] = src["a.cuh"].replace("{\n", "{\n    pdl_wait();\n", 1)
    (_, head), = list(_bodies(src, "k_demo"))
    assert "pdl_wait();" in head
