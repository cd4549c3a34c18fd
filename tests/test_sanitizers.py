"""Host C/C++ code under gcc's address and undefined-behaviour sanitizers (CPU).

compute-sanitizer does not run here, so the host-side code is checked this way:
* the oracle's C restatement (oracle/swe_oracle.c), FP64 and FP32, driven
  through eval_rhs, three RK4 steps and the invariants on a synthetic grid;
* the library's host RCM ordering (csrc/host_layout.cu, plain host C++),
  on a valid stencil graph (the result must be a permutation) and on one with
  an out-of-range index (it must report SWE_ERR_INDEX without reading past).
Any sanitizer finding aborts the program (-fno-sanitize-recover=all).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-g", "-O1"]

ORACLE_DRIVER = r"""
#include <stdio.h>
#include "swe_oracle.c"

static unsigned long long s = 88172645463325252ULL;
static double rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (double)(s >> 11) / 9007199254740992.0; }

int main(void) {
    enum { N = 300, NNBR = 31, STRIDE = 32 };
    static int idx[N * STRIDE];
    static real Dx[N * STRIDE], Dy[N * STRIDE], Dz[N * STRIDE], L[N * STRIDE];
    static real x[N], y[N], z[N], f[N], ghm[N], pu[3 * N], pv[3 * N], pw[3 * N], gg[3 * N];
    static real K[4 * N], F[4 * N], H[4 * N];
    for (int i = 0; i < N; i++) {
        for (int j = 0; j < STRIDE; j++) {
            idx[i * STRIDE + j] = j == 0 ? i : (int)(rnd() * N) % N;
            Dx[i * STRIDE + j] = (real)(1e-6 * (rnd() - 0.5));
            Dy[i * STRIDE + j] = (real)(1e-6 * (rnd() - 0.5));
            Dz[i * STRIDE + j] = (real)(1e-6 * (rnd() - 0.5));
            L[i * STRIDE + j] = (real)(1e-9 * (rnd() - 0.5));
        }
        x[i] = (real)rnd(); y[i] = (real)rnd(); z[i] = (real)rnd(); f[i] = (real)1e-4; ghm[i] = (real)(100.0 * rnd());
        for (int c = 0; c < 3; c++) {
            pu[3 * i + c] = (real)rnd(); pv[3 * i + c] = (real)rnd(); pw[3 * i + c] = (real)rnd();
            gg[3 * i + c] = (real)(1e-3 * rnd());
        }
        for (int c = 0; c < 4; c++) K[4 * i + c] = H[4 * i + c] = (real)(c == 3 ? 5960.0 * (1 + 1e-3 * rnd()) : 20.0 * rnd());
    }
    OracleGrid g = {N, NNBR, STRIDE, (real)(9.80616 * 5960.0), (real)100.0, idx, Dx, Dy, Dz, L,
                    x, y, z, f, ghm, pu, pv, pw, gg};
    oracle_eval_rhs(&g, K, F);
    oracle_run(&g, H, 3);
    double inv[2];
    oracle_invariants(&g, H, 1, inv);
    for (int t = 0; t < 4 * N; t++)
        if (!(F[t] == F[t]) || !(H[t] == H[t])) { printf("nan at %d\n", t); return 1; }
    printf("ok %g %g\n", inv[0], inv[1]);
    return 0;
}
"""

RCM_DRIVER = r"""
#include <cstdarg>
#include <cstdio>
#include <vector>
namespace swe {
void set_error(const char* fmt, ...) { va_list ap; va_start(ap, fmt); vfprintf(stderr, fmt, ap); va_end(ap); }
void count_launch(long long) {}
}
extern "C" int swe_host_rcm_mapping(int n, int nnbr, const int* idx, int* mapping);

int main() {
    const int n = 500, nnbr = 9;
    const int off[nnbr] = {0, 1, -1, 2, -2, 17, -17, 31, -31};
    std::vector<int> idx(n * nnbr), map(n, -1), seen(n, 0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < nnbr; ++j) idx[i * nnbr + j] = ((i + off[j]) % n + n) % n;
    if (swe_host_rcm_mapping(n, nnbr, idx.data(), map.data()) != 0) return 2;
    for (int i = 0; i < n; ++i) {
        if (map[i] < 0 || map[i] >= n || seen[map[i]]++) { std::printf("not a permutation at %d\n", i); return 3; }
    }
    idx[123 * nnbr + 4] = n + 7;                    // out of range: reported, never read through
    if (swe_host_rcm_mapping(n, nnbr, idx.data(), map.data()) != 5) return 4;
    std::printf("ok\n");
    return 0;
}
"""


def _compilers():
    cc, cxx = shutil.which("gcc"), shutil.which("g++")
    if not cc or not cxx:
        pytest.skip("no gcc/g++")
    return cc, cxx


@pytest.mark.parametrize("prec", ["ORACLE_FP64", "ORACLE_FP32"])
def test_oracle_restatement_under_sanitizers(tmp_path, prec):
    cc, _ = _compilers()
    src = tmp_path / "oracle_driver.c"
    src.write_text(ORACLE_DRIVER)
    exe = tmp_path / "oracle_driver"
    subprocess.run([cc, "-std=c99", *SAN, f"-D{prec}", "-I", os.path.join(ROOT, "oracle"), str(src), "-o", str(exe),
                    "-lm"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr[-3000:]


def test_host_rcm_under_sanitizers(tmp_path):
    _, cxx = _compilers()
    drv = tmp_path / "rcm_driver.cpp"
    drv.write_text(RCM_DRIVER)
    exe = tmp_path / "rcm_driver"
    cuda_inc = "/usr/local/cuda/include"
    if not os.path.isdir(cuda_inc):
        pytest.skip("CUDA headers not found")
    subprocess.run([cxx, "-std=c++17", *SAN, "-w", "-I", cuda_inc, "-I", os.path.join(ROOT, "include"),
                    "-x", "c++", os.path.join(ROOT, "rbf-fd-swe_b200", "csrc", "host_layout.cu"),
                    "-x", "none", str(drv), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr[-3000:]
