"""The step kernels' division by the spacing (div4 in ouc_b200/csrc/fd_step.cuh:
Markstein-corrected reciprocal, and the scaled single-precision form for
dividends below the tiny-quotient threshold) equals IEEE single division
(__fdiv_rn) bit for bit: every tiny dividend of both signs, exhaustively,
plus a strided sample of all normal dividends, for the spacings of the
workloads and a few more.  Compiled from the kernel header with nvcc and run
on the GPU (a few hundred million divisions)."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <cstdio>
#include <cstring>
#include "fd_step.cuh"
using namespace ouc;

__global__ void k_check(float h, float r, unsigned lo, unsigned hi, unsigned stride, unsigned long long* bad,
                        unsigned* first) {
    const Div d = make_div(h, r);
    const unsigned long long n = (hi - lo + stride - 1) / stride;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned u = lo + (unsigned)(i * stride);
        const float x = __uint_as_float(u);
        const float4 q = div4(make_float4(x, -x, x, -x), d);
        const float e = __fdiv_rn(x, h), en = __fdiv_rn(-x, h);
        if (__float_as_uint(q.x) != __float_as_uint(e) || __float_as_uint(q.y) != __float_as_uint(en)) {
            atomicAdd(bad, 1ull);
            atomicCAS(first, 0u, u);
        }
    }
}

int main() {
    const float hs[] = {5.f, 4.f, 10.f, 2.f, 8.f, 20.f, 2.5f, 12.5f, 1.f, 3.f, 7.f, 0.5f, 256.f, 100.f, 6.25f, 15.f};
    unsigned long long* d_bad;
    unsigned* d_first;
    cudaMalloc(&d_bad, 8);
    cudaMalloc(&d_first, 4);
    unsigned long long total = 0, count = 0;
    for (float h : hs) {
        volatile float one = 1.f;
        const float r = one / h;
        const float T = nextafterf(0x1p-124f * (float)((double)h * (1.0 + 0x1p-22)), INFINITY);
        unsigned tb;
        memcpy(&tb, &T, 4);
        // every tiny dividend (and 4096 above the threshold), then a strided sample of the normal ones
        const unsigned ranges[2][3] = {{1u, tb + 4096u, 1u}, {tb, 0x7f000000u, 4099u}};
        for (auto& rg : ranges) {
            cudaMemset(d_bad, 0, 8);
            cudaMemset(d_first, 0, 4);
            k_check<<<148 * 8, 256>>>(h, r, rg[0], rg[1], rg[2], d_bad, d_first);
            unsigned long long bad = 0;
            unsigned first = 0;
            if (cudaMemcpy(&bad, d_bad, 8, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
            cudaMemcpy(&first, d_first, 4, cudaMemcpyDeviceToHost);
            count += (rg[1] - rg[0] + rg[2] - 1) / rg[2];
            if (bad) printf("h=%g: %llu mismatches, first dividend bits 0x%08x\n", h, bad, first);
            total += bad;
        }
    }
    printf("%llu %llu\n", count, total);
    return total != 0;
}
"""


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc")
def test_division_equals_ieee(tmp_path):
    src = tmp_path / "div.cu"
    src.write_text(SRC)
    exe = tmp_path / "div"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "ouc_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    count, bad = map(int, r.stdout.split()[-2:])
    assert r.returncode == 0 and bad == 0 and count > 500_000_000, r.stdout
