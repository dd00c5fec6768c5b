"""Writes the reference's kernel table header with the CUDA rows added -- the
edit INTEGRATION.md section 2 tells a maintainer to make to
src/KernelFunctions.h -- into a build directory, so that the reference's own
driver (src/Main.c) can be linked against liblbmb200.so without touching the
reference sources. TEST INFRASTRUCTURE: oracle/Makefile runs it for
oracle/_ref/lbmbenchk-cuda, which only tests run.

    python oracle/kernel_table_cuda.py <reference src/KernelFunctions.h> <output path>

The rows are appended after the reference's own rows of g_kernels, and
lbm_b200.h is included after the reference's kernel headers (it then reuses
the reference's LatticeDesc/KernelData/CaseData/Parameters).
"""
import re
import sys

ROWS = [
    ("cuda-aa-soa", "D3Q19CudaAaInit_AaSoA", "D3Q19CudaAaDeinit_AaSoA"),
    ("cuda-list-aa-pv-soa", "D3Q19CudaListAaPvInit_PushSoA", "D3Q19CudaListAaPvDeinit_PushSoA"),
    ("cuda-list-pull-split-nt-1s-soa", "D3Q19CudaListPullSplitNt1SInit_PullSoA",
     "D3Q19CudaListPullSplitNtDeinit_PullSoA"),
    ("cuda-list-pull-split-nt-2s-soa", "D3Q19CudaListPullSplitNt2SInit_PullSoA",
     "D3Q19CudaListPullSplitNtDeinit_PullSoA"),
    ("cuda-list-aa-soa", "D3Q19CudaListAaInit_PushSoA", "D3Q19CudaListAaDeinit_PushSoA"),
    ("cuda-list-aa-ria-soa", "D3Q19CudaListAaRiaInit_PushSoA", "D3Q19CudaListAaRiaDeinit_PushSoA"),
    ("cuda-list-push-soa", "D3Q19CudaListInit_PushSoA", "D3Q19CudaListDeinit_PushSoA"),
    ("cuda-list-pull-soa", "D3Q19CudaListInit_PullSoA", "D3Q19CudaListDeinit_PullSoA"),
    ("cuda-push-soa", "D3Q19CudaInit_PushSoA", "D3Q19CudaDeinit_PushSoA"),
    ("cuda-pull-soa", "D3Q19CudaInit_PullSoA", "D3Q19CudaDeinit_PullSoA"),
]


def main():
    src, out = sys.argv[1], sys.argv[2]
    text = open(src).read()
    # lbm_b200.h right before the table's struct definition
    anchor = "typedef struct KernelFunctions_"
    if anchor not in text:
        raise SystemExit("kernel table struct not found in %s" % src)
    text = text.replace(anchor, '#include "lbm_b200.h"\n\n' + anchor, 1)
    # the rows before the closing brace of g_kernels
    m = re.search(r"KernelFunctions\s+g_kernels\s*\[\]\s*=\s*\{", text)
    if not m:
        raise SystemExit("g_kernels not found in %s" % src)
    end = text.index("};", m.end())
    body = text[m.end():end].rstrip()
    rows = "".join("\n\t{\n\t\t.Name   = \"%s\",\n\t\t.Init   = %s,\n\t\t.Deinit = %s\n\t}," % r for r in ROWS)
    sep = "" if body.endswith(",") else ","
    text = text[:m.end()] + body + sep + rows + "\n" + text[end:]
    with open(out, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main()
