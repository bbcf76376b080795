"""The opening pass of Reset_states_horizontal/_vertical (support_funcs.cu:75-186) as the
column/row resets run it (CPU model, no GPU).

The reference runs the pass serially over k = 2..L: when t_z[k] > z[k], a neighbour whose
mask is 1 is opened with t_z[k] and FS[k].  The library's k_reset tests every cell of the
line at once (t_z > z, a mask-1 neighbour) and runs only the passing cells in increasing
order, each followed by its cascade (a cell opened to the right is the next iteration and
carries the opener's t_z).  This model of that order must leave exactly the state of the
serial loop; the kernel itself is checked against the oracle by the GPU parity tests."""
import numpy as np


def serial_pass(K, T, Z, F, L):
    K, T, F = K.copy(), T.copy(), F.copy()
    for k in range(2, L + 1):
        if T[k] > Z[k]:
            if K[k - 1] == 1:
                T[k - 1], K[k - 1], F[k - 1] = T[k], 0, F[k]
            if K[k + 1] == 1:
                T[k + 1], K[k + 1], F[k + 1] = T[k], 0, F[k]
    return K, T, F


def event_pass(K0, T0, Z, F0, L):
    K, T, F = K0.copy(), T0.copy(), F0.copy()
    open_ = np.flatnonzero(K0 != 2)
    lo, hi = open_.min(), open_.max()
    k0, k1 = max(lo - 1, 0), min(hi + 1, L + 2)  # the staged span, widened by one cell

    def khv(k):
        return K[k] if k0 <= k <= k1 else 2

    events = [k for k in range(k0, k1 + 1)
              if 2 <= k <= L and T0[k] > Z[k] and (khv(k - 1) == 1 or khv(k + 1) == 1)]
    kb = min(k1, L)
    done = -1
    for m in events:
        if m <= done:
            continue  # already run inside a cascade
        t, f = T[m], F[m]
        act = True
        while True:
            done = m
            if not act:
                break
            right = False
            if khv(m - 1) == 1:
                T[m - 1], K[m - 1], F[m - 1] = t, 0, f
            if khv(m + 1) == 1:
                T[m + 1], K[m + 1], F[m + 1] = t, 0, f
                right = True
            if not right or m + 1 > kb:
                break
            m += 1
            act = t > Z[m]
    return K, T, F


def test_event_order_equals_serial_pass():
    rng = np.random.default_rng(0)
    for trial in range(4000):
        L = int(rng.integers(3, 40))
        n = L + 3
        K = rng.choice([0, 1, 2], size=n, p=[0.35, 0.45, 0.2])
        if trial % 3 == 0:
            K[:rng.integers(0, n)] = 2
        if (K != 2).sum() == 0:
            K[n // 2] = 0
        T = rng.normal(size=n)
        Z = rng.normal(size=n) - rng.uniform(0, 1)
        F = rng.normal(size=n)
        a = serial_pass(K, T, Z, F, L)
        b = event_pass(K, T, Z, F, L)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), (trial, K)
