"""The host half of the Anderson acceleration (csrc/anderson.h) against the
numpy formulas of oracle/port.py, without a GPU.

A small C++ driver compiles the header with g++, restates on the CPU what the
aa_update / aa_mix kernels compute (same column ring, same dot layout) and
runs the mixing on linear fixed-point maps w -> A w + c for two instances
with different memories in one allocation, with mu changes and a residual
jump that trips the restart rule.  The numpy side replays the port's history
rule (reset on a mu change or when |f| more than doubles, at most m columns)
on the same maps; the trajectories must agree to rounding."""
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "anderson.h"

int main() {
    int B, N, S;
    if (std::scanf("%d %d %d", &B, &N, &S) != 3) return 1;
    std::vector<int> mem(B);
    int M = 0;
    for (int b = 0; b < B; b++) { std::scanf("%d", &mem[b]); if (mem[b] > M) M = mem[b]; }
    std::vector<double> A((size_t)B * N * N), c((size_t)B * N), w((size_t)B * N);
    for (auto& v : A) std::scanf("%lf", &v);
    for (auto& v : c) std::scanf("%lf", &v);
    for (auto& v : w) std::scanf("%lf", &v);
    std::vector<int> muchg((size_t)S * B), kick((size_t)S * B);
    for (auto& v : muchg) std::scanf("%d", &v);
    for (auto& v : kick) std::scanf("%d", &v);
    // device buffers of the kernels, one column of N rows per instance
    std::vector<double> fprev((size_t)B * N, 0.0), gprev((size_t)B * N, 0.0);
    std::vector<double> dF((size_t)M * B * N, 0.0), dG((size_t)M * B * N, 0.0);
    v2g::AndersonState aa(B, M);
    for (int k = 0; k < S; k++) {
        std::vector<double> g((size_t)B * N);
        for (int b = 0; b < B; b++)
            for (int i = 0; i < N; i++) {
                double s = c[(size_t)b * N + i];
                for (int j = 0; j < N; j++) s += A[((size_t)b * N + i) * N + j] * w[(size_t)b * N + j];
                if (kick[(size_t)k * B + b]) s += 100.0;  // a step that went the wrong way
                g[(size_t)b * N + i] = s;
            }
        std::vector<double> dots((size_t)(2 * M + 1) * B, 0.0);
        for (int b = 0; b < B; b++) {
            const int md = aa.begin(b, mem[b], muchg[(size_t)k * B + b] != 0);
            if (!md) continue;
            const int s = aa.slot[b];
            double ff = 0.0;
            std::vector<double> acc(2 * M, 0.0);
            for (int i = 0; i < N; i++) {
                const size_t t = (size_t)b * N + i;
                const double f = g[t] - w[t];
                if (md == 2) {
                    const double df = f - fprev[t];
                    dF[(size_t)s * B * N + t] = df;
                    dG[(size_t)s * B * N + t] = g[t] - gprev[t];
                    for (int j = 0; j < M; j++) {
                        const double dj = (j == s) ? df : dF[(size_t)j * B * N + t];
                        acc[2 * j] += df * dj;
                        acc[2 * j + 1] += dj * f;
                    }
                }
                ff += f * f;
                fprev[t] = f;
                gprev[t] = g[t];
            }
            for (int q = 0; q < 2 * M; q++) dots[(size_t)q * B + b] = acc[q];
            dots[(size_t)(2 * M) * B + b] = ff;
        }
        std::vector<double> gamma((size_t)B * M, 0.0);
        for (int b = 0; b < B; b++) {
            const bool mix = aa.finish(b, mem[b], dots, &gamma[(size_t)b * M]);
            for (int i = 0; i < N; i++) {
                const size_t t = (size_t)b * N + i;
                double v = g[t];
                if (mix)
                    for (int j = 0; j < M; j++)
                        if (gamma[(size_t)b * M + j] != 0.0) v -= gamma[(size_t)b * M + j] * dG[(size_t)j * B * N + t];
                w[t] = v;
            }
        }
        for (size_t t = 0; t < w.size(); t++) std::printf("%.17g\n", w[t]);
    }
    return 0;
}
"""


def _numpy_trajectory(A, c, w0, m, muchg, kick):
    """The port's Anderson rule (oracle/port.py solve) on w -> A w + c."""
    hw, hf, fprev = [], [], None
    w, out = w0.copy(), []
    for k in range(len(muchg)):
        g = A @ w + c + (100.0 if kick[k] else 0.0)
        f = g - w
        fn = np.linalg.norm(f)
        if muchg[k] or (fprev is not None and fn > 2.0 * fprev):
            hw, hf = [], []
        fprev = fn
        hw.append(w)
        hf.append(f)
        if len(hw) > m + 1:
            hw.pop(0)
            hf.pop(0)
        if len(hf) >= 2:
            dF = np.stack([hf[i + 1] - hf[i] for i in range(len(hf) - 1)], axis=1)
            dG = np.stack([(hw[i + 1] + hf[i + 1]) - (hw[i] + hf[i]) for i in range(len(hf) - 1)], axis=1)
            Mx = dF.T @ dF
            Mx = Mx + (1e-10 * np.trace(Mx) + 1e-300) * np.eye(Mx.shape[0])
            g = g - dG @ np.linalg.solve(Mx, dF.T @ f)
        w = g
        out.append(w.copy())
    return np.array(out)


def test_anderson_host_state_matches_port_rule():
    rng = np.random.default_rng(5)
    B, N, S = 2, 12, 24
    mem = [3, 2]
    As, cs, ws = [], [], []
    for _ in range(B):
        Q, _ = np.linalg.qr(rng.standard_normal((N, N)))
        As.append(Q @ np.diag(rng.uniform(0.3, 0.95, N)) @ Q.T)
        cs.append(rng.standard_normal(N))
        ws.append(rng.standard_normal(N))
    muchg = np.zeros((S, B), dtype=int)
    muchg[9, 0] = 1
    muchg[14, 1] = 1
    kick = np.zeros((S, B), dtype=int)
    kick[17, 0] = 1  # |f| jumps: the history restarts
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "drv.cpp"), os.path.join(d, "drv")
        with open(src, "w") as fh:
            fh.write(DRIVER)
        subprocess.run(["g++", "-std=c++17", "-O1", "-w", "-I", os.path.join(ROOT, "v2rdm_casscf_b200", "csrc"), src, "-o",
                        exe], check=True)
        lines = [f"{B} {N} {S}", " ".join(map(str, mem))]
        lines += [" ".join("%.17g" % v for v in a.ravel()) for a in As]
        lines += [" ".join("%.17g" % v for v in a) for a in cs]
        lines += [" ".join("%.17g" % v for v in a) for a in ws]
        lines += [" ".join(map(str, muchg.ravel())), " ".join(map(str, kick.ravel()))]
        out = subprocess.run([exe], input="\n".join(lines), capture_output=True, text=True, check=True).stdout
    got = np.array([float(v) for v in out.split()]).reshape(S, B, N)
    for b in range(B):
        want = _numpy_trajectory(As[b], cs[b], ws[b], mem[b], muchg[:, b], kick[:, b])
        scale = np.abs(want).max(axis=1, keepdims=True)
        assert np.all(np.abs(got[:, b, :] - want) <= 1e-9 * scale + 1e-12)
    # the mixing did something: the trajectory differs from the plain iteration
    plain = ws[0].copy()
    for _ in range(8):
        plain = As[0] @ plain + cs[0]
    assert np.abs(got[7, 0] - plain).max() > 1e-6
