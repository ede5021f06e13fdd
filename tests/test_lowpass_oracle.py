"""The oracle's restatement of the 2D spectral low-pass (cuda/kernels/gaussian.hpp,
lowpass.hpp): known answers and the LOWPASS format, on the CPU."""
import math
import pickle

import numpy as np

import pfc_oracle as O


def test_lowpass_header_is_the_protocol0_pickle_it_claims():
    text = O.lowpass_text(np.zeros((12, 9), np.complex64), 16, 12, 12.566, 9.42, np.float32)
    tag, n, rest = text.split(b"\n", 2)
    assert tag == b"LOWPASS"
    head = rest[: int(n)]
    assert head.endswith(b"d.\n")
    d = pickle.loads(head)
    assert d["n0"] == 16 and d["n1"] == 12
    assert abs(d["l0"] - 12.566) < 1e-6 and abs(d["l1"] - 9.42) < 1e-6
    assert rest[int(n):] == b""  # an all-zero spectrum has no entries


def test_lowpass_entries_order_threshold_and_format():
    nx, ny = 8, 4
    sp = np.zeros((ny, nx // 2 + 1), np.complex128)
    sp[0, 0] = 2.5
    sp[3, 0] = 1e-3 + 1e-4j       # |a|^2 = 1.01e-6 > 1e-6: written
    sp[1, 2] = 0.5e-3 + 0.5e-3j   # |a|^2 = 5e-7: dropped
    sp[2, 4] = -1234567.0 - 1e-8j
    body = O.lowpass_text(sp, nx, ny, 1.0, 1.0, np.float64).split(b"d.\n", 1)[1].decode()
    assert body.splitlines() == ["0 0 2.5 0", "0 3 0.001 0.0001", "4 2 -1.23457e+06 -1e-08"]


def test_gaussian_filter_limits():
    shape, lens, hh = (32, 24, 1), (25.0, 20.0, 1.0), (0.78, 0.83, 1.0)
    g = O.gaussian_init(shape, lens, hh, 2.0, np.float64)
    assert g[0, 0, 0] == 1.0 + 0.0j
    np.testing.assert_allclose(g.real + g.imag, 1.0, atol=1e-15)
    # e depends on |k| through the spacings: +-ky give the same value
    np.testing.assert_array_equal(g[0, 1, :], g[0, -1, :])
    k0 = 2 * math.pi / lens[0]
    assert abs(g[0, 0, 1].real - math.exp(-0.5 * (1.1 * 2.0 * hh[0] * k0) ** 2)) < 1e-15


def test_amplitude_of_a_cosine_known_answer_oracle():
    nx, ny = 64, 16
    lens, hh = (64 * 0.8, 16 * 0.8, 1.0), (0.8, 0.8, 1.0)
    x = np.arange(nx) * lens[0] / nx
    m, A = 5, 1.3
    q = 2 * math.pi * m / lens[0]
    psi = np.broadcast_to(A * np.cos(q * x), (1, ny, nx)).copy()
    g = O.gaussian_init((nx, ny, 1), lens, hh, 1.0, np.float64)
    amp, low = O.amplitude_lowpass(O.r2c(psi), g, (nx, ny, 1))
    eq, e2q = g[0, 0, m].real, g[0, 0, 2 * m].real
    want = (1 - eq) ** 2 * A * A / 2 * (1 + e2q * np.cos(2 * q * x))
    np.testing.assert_allclose(amp[0], np.broadcast_to(want, (ny, nx)), atol=1e-13)
    assert abs(low[0, 0, 0].real - (1 - eq) ** 2 * A * A / 2 * nx * ny) < 1e-9
