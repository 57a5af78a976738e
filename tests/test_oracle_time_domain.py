"""TIME_DOMAIN ProcessDirect restatement (oracle/tan_cpu_ref.cpp) against an
independent float64 numpy statement of the reference's algorithm
(tan/tanlibrary/src/TrueAudioNext/convolution/ConvolutionImpl.cpp:721-762
ProcessDirect, :2757-2782 ovlTimeDomainCPU): a circular history of
N = nextpow2(L) samples per channel; each call first writes all its n inputs
(n clamped to N) at the running position, then out[j] = sum over taps k in
[first, last) of hist[(pos + j - k) mod N] * ir[k]; the position advances by n.
When n + L - 1 <= N this is the linear convolution of the call stream.
Tolerance: max error <= 1e-5 of the output RMS (the restatement accumulates
up to N float32 products per sample in the reference's order)."""
import numpy as np
import pytest

from oracle import fp64, ref
from tests import helpers as H


def nextpow2(n):
    p = 1
    while p < n:
        p <<= 1
    return p


class TdStatement:
    def __init__(self, L, C):
        self.N = nextpow2(L)
        self.hist = np.zeros((C, self.N))
        self.pos = 0

    def call(self, ir, x, nz=None):
        C, n = x.shape
        N = self.N
        n = min(n, N)
        out = np.zeros((C, n))
        for c in range(C):
            first, last = (0, N) if nz is None else (nz[2 * c], nz[2 * c + 1])
            self.hist[c, (self.pos + np.arange(n)) % N] = x[c, :n]
            k = np.arange(first, last)
            for j in range(n):
                out[c, j] = np.dot(self.hist[c, (self.pos + j - k) % N], ir[c, first:last].astype(np.float64))
        self.pos += n
        return out, n


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-30, np.sqrt(np.mean(b * b))))


@pytest.mark.parametrize("L,calls", [(1000, [256, 700, 1024, 64, 1500]), (300, [512, 100, 512, 17])])
def test_restatement_matches_statement(L, calls):
    C = 2
    g = H.rng(L + len(calls))
    td = ref.RefTimeDomain(L, C)
    st = TdStatement(L, C)
    N = st.N
    for i, n in enumerate(calls):
        ir = np.zeros((C, N), np.float32)
        ir[:, :L] = H.irs(g, C, L, (0.05, 0.2))
        x = H.noise(g, C, n)
        nz = None if i % 2 == 0 else [3, L - 5, 0, L // 2]
        if nz is not None:
            for c in range(C):  # taps outside [first, last) must not count
                ir[c, :nz[2 * c]] = 7.0
                ir[c, nz[2 * c + 1]:] = -7.0
        rc, y, done = td.process_direct(ir, x, nz)
        exp, n_exp = st.call(ir, x.astype(np.float64), nz)
        assert rc == 0 and done == n_exp == min(n, N)
        assert _rel(y[:, :done].astype(np.float64), exp) < 1e-5, (i, _rel(y[:, :done], exp))
    td.close()


def test_restatement_is_linear_convolution_when_history_fits():
    """Fixed IR, calls of n with n + L - 1 <= N: the stream output equals x * h."""
    C, L, n, ncalls = 2, 700, 256, 12
    g = H.rng(77)
    N = nextpow2(L)
    assert n + L - 1 <= N
    h = H.irs(g, C, L, (0.05, 0.2))
    ir = np.zeros((C, N), np.float32)
    ir[:, :L] = h
    x = H.noise(g, C, n * ncalls)
    td = ref.RefTimeDomain(L, C)
    y = np.zeros((C, n * ncalls), np.float32)
    for i in range(ncalls):
        rc, yi, done = td.process_direct(ir, np.ascontiguousarray(x[:, i * n:(i + 1) * n]))
        assert rc == 0 and done == n
        y[:, i * n:(i + 1) * n] = yi
    td.close()
    for c in range(C):
        assert fp64.error_db(y[c], fp64.conv_fp64(x[c], h[c])) < -120
