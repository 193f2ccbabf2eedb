"""1D summation-by-parts operators (oracle; test infrastructure only).

Restates source/spmat.cpp:310-627 of the reference.  All matrices are dense
numpy arrays of shape (N, N); the 2D assembly converts them to sparse.
"""
import numpy as np


def sbp_spmat(order, N, scale, compat="fullyCompatible"):
    """H, Hinv, D1, D1int, BS for one direction (spmat.cpp:310-491).

    ``scale`` is 1/h.  Returns a dict of dense arrays.  For N == 1 only H is
    set (to the identity) and the rest are zero, as in spmat.cpp:321-324.
    """
    H = np.zeros((N, N)); Hinv = np.zeros((N, N))
    D1int = np.zeros((N, N)); BS = np.zeros((N, N))
    if N == 1:
        H[0, 0] = 1.0
        return dict(H=H, Hinv=Hinv, D1=D1int.copy(), D1int=D1int, BS=BS)
    if order == 2:
        # spmat.cpp:330-380
        H[:] = np.eye(N); H[0, 0] = 0.5; H[N - 1, N - 1] = 0.5
        H *= 1.0 / scale
        for i in range(N):
            Hinv[i, i] = 1.0 / H[i, i]
        D1int[0, 0] = -1.0 * scale; D1int[0, 1] = scale
        for i in range(1, N - 1):
            D1int[i, i - 1] = -0.5 * scale
            D1int[i, i + 1] = 0.5 * scale
        D1int[N - 1, N - 1] = scale; D1int[N - 1, N - 2] = -1 * scale
        D1 = D1int.copy()
        if compat == "fullyCompatible":
            BS[0, 0] = -D1int[0, 0]; BS[0, 1] = -D1int[0, 1]
            BS[N - 1, N - 2] = D1int[N - 1, N - 2]; BS[N - 1, N - 1] = D1int[N - 1, N - 1]
        elif compat == "compatible":
            BS[0, 0] = 1.5 * scale; BS[0, 1] = -2.0 * scale; BS[0, 2] = 0.5 * scale
            BS[N - 1, N - 3] = 0.5 * scale; BS[N - 1, N - 2] = -2.0 * scale; BS[N - 1, N - 1] = 1.5 * scale
            D1[0, 0] = -BS[0, 0]; D1[0, 1] = -BS[0, 1]; D1[0, 2] = -BS[0, 2]
            D1[N - 1, N - 3] = BS[N - 1, N - 3]; D1[N - 1, N - 2] = BS[N - 1, N - 2]
            D1[N - 1, N - 1] = BS[N - 1, N - 1]
        else:
            raise ValueError("SBP type not understood")
        return dict(H=H, Hinv=Hinv, D1=D1, D1int=D1int, BS=BS)
    if order == 4:
        # spmat.cpp:382-491
        if not N > 8:
            raise ValueError("N must be > 8 for 4th order SBP")
        H[:] = np.eye(N)
        for i, v in enumerate((17.0 / 48.0, 59.0 / 48.0, 43.0 / 48.0, 49.0 / 48.0)):
            H[i, i] = v
            H[N - 1 - i, N - 1 - i] = v
        H *= 1.0 / scale
        for i in range(N):
            Hinv[i, i] = 1.0 / H[i, i]
        for i in range(4, N - 4):
            hi = Hinv[i, i]
            D1int[i, i - 2] = 1.0 / 12.0 * hi
            D1int[i, i - 1] = -2.0 / 3.0 * hi
            D1int[i, i + 1] = 2.0 / 3.0 * hi
            D1int[i, i + 2] = -1.0 / 12.0 * hi
        h = lambda i: Hinv[i, i]
        # closure rows (spmat.cpp:409-446)
        D1int[0, 0] = -1.0 / 2.0 * h(0); D1int[0, 1] = 59.0 / 96.0 * h(0)
        D1int[0, 2] = -1.0 / 12.0 * h(0); D1int[0, 3] = -1.0 / 32.0 * h(0)
        D1int[1, 0] = -59.0 / 96.0 * h(1); D1int[1, 2] = 59.0 / 96.0 * h(1)
        D1int[2, 0] = 1.0 / 12.0 * h(2); D1int[2, 1] = -59.0 / 96.0 * h(2)
        D1int[2, 3] = 59.0 / 96.0 * h(2); D1int[2, 4] = -1.0 / 12.0 * h(2)
        D1int[3, 0] = 1.0 / 32.0 * h(3); D1int[3, 2] = -59.0 / 96.0 * h(3)
        D1int[3, 4] = 2.0 / 3.0 * h(3); D1int[3, 5] = -1.0 / 12.0 * h(3)
        n = N
        D1int[n - 1, n - 1] = 1.0 / 2.0 * h(n - 1); D1int[n - 1, n - 2] = -59.0 / 96.0 * h(n - 1)
        D1int[n - 1, n - 3] = 1.0 / 12.0 * h(n - 1); D1int[n - 1, n - 4] = 1.0 / 32.0 * h(n - 1)
        D1int[n - 2, n - 1] = 59.0 / 96.0 * h(n - 2); D1int[n - 2, n - 3] = -59.0 / 96.0 * h(n - 2)
        D1int[n - 3, n - 1] = -1.0 / 12.0 * h(n - 3); D1int[n - 3, n - 2] = 59.0 / 96.0 * h(n - 3)
        D1int[n - 3, n - 4] = -59.0 / 96.0 * h(n - 3); D1int[n - 3, n - 5] = 1.0 / 12.0 * h(n - 3)
        D1int[n - 4, n - 1] = -1.0 / 32.0 * h(n - 4); D1int[n - 4, n - 3] = 59.0 / 96.0 * h(n - 4)
        D1int[n - 4, n - 5] = -2.0 / 3.0 * h(n - 4); D1int[n - 4, n - 6] = 1.0 / 12.0 * h(n - 4)
        D1 = D1int.copy()
        if compat == "fullyCompatible":
            BS[0, 0] = 24.0 / 17.0 * scale; BS[0, 1] = -59.0 / 34.0 * scale
            BS[0, 2] = 4.0 / 17.0 * scale; BS[0, 3] = 3.0 / 34.0 * scale
            BS[n - 1, n - 1] = 24.0 / 17.0 * scale; BS[n - 1, n - 2] = -59.0 / 34.0 * scale
            BS[n - 1, n - 3] = 4.0 / 17.0 * scale; BS[n - 1, n - 4] = 3.0 / 34.0 * scale
        elif compat == "compatible":
            # the last row of the reference omits ``scale`` (spmat.cpp:463)
            BS[0, 0] = 11.0 / 6.0 * scale; BS[0, 1] = -3.0 * scale
            BS[0, 2] = 1.5 * scale; BS[0, 3] = -1.0 / 3.0 * scale
            BS[n - 1, n - 1] = 11.0 / 6.0; BS[n - 1, n - 2] = -3.0
            BS[n - 1, n - 3] = 1.5; BS[n - 1, n - 4] = -1.0 / 3.0
            D1[0, 0] = -BS[0, 0]; D1[0, 1] = -BS[0, 1]; D1[0, 2] = -BS[0, 2]; D1[0, 3] = -BS[0, 3]
            # the reference sets (N-1, N-4) twice and never (N-1, N-3) (spmat.cpp:466)
            D1[n - 1, n - 4] = BS[n - 1, n - 4]
            D1[n - 1, n - 2] = BS[n - 1, n - 2]; D1[n - 1, n - 1] = BS[n - 1, n - 1]
        else:
            raise ValueError("SBP type not understood")
        return dict(H=H, Hinv=Hinv, D1=D1, D1int=D1int, BS=BS)
    raise ValueError("order not understood")


def sbp_spmat2(N, scale):
    """D2 and C2 for the order-2 R term (spmat.cpp:494-544)."""
    D2 = np.zeros((N, N)); C2 = np.zeros((N, N))
    if N == 1:
        return D2, C2
    s2 = scale * scale
    D2[0, 0] = s2; D2[0, 1] = -2.0 * s2; D2[0, 2] = s2
    for i in range(1, N - 1):
        D2[i, i - 1] = s2; D2[i, i] = -2.0 * s2; D2[i, i + 1] = s2
    D2[N - 1, N - 3] = s2; D2[N - 1, N - 2] = -2.0 * s2; D2[N - 1, N - 1] = s2
    C2[:] = np.eye(N); C2[0, 0] = 0; C2[N - 1, N - 1] = 0
    return D2, C2


def sbp_spmat4(N, scale):
    """D3, D4, C3, C4 for the order-4 R term (spmat.cpp:547-627).

    ``scale`` is accepted for signature parity; the reference does not use it
    (the 1/h factors are applied by the caller).
    """
    D3 = np.zeros((N, N)); D4 = np.zeros((N, N)); C3 = np.zeros((N, N)); C4 = np.zeros((N, N))
    if N == 1:
        return D3, D4, C3, C4
    n = N
    for r in (0, 1):
        D3[r, 0:4] = (-1, 3, -3, 1)
    D3[2, 0] = -185893.0 / 301051.0
    D3[2, 1] = 79000249461.0 / 54642863857.0
    D3[2, 2] = -33235054191.0 / 54642863857.0
    D3[2, 3] = -36887526683.0 / 54642863857.0
    D3[2, 4] = 26183621850.0 / 54642863857.0
    D3[2, 5] = -4386.0 / 181507.0
    for i in range(3, n - 4):
        D3[i, i - 1] = -1.0; D3[i, i] = 3; D3[i, i + 1] = -3; D3[i, i + 2] = 1.0
    D3[n - 3, n - 1] = -D3[2, 0]; D3[n - 3, n - 2] = -D3[2, 1]; D3[n - 3, n - 3] = -D3[2, 2]
    D3[n - 3, n - 4] = -D3[2, 3]; D3[n - 3, n - 5] = -D3[2, 4]; D3[n - 3, n - 6] = -D3[2, 5]
    D3[n - 2, n - 4:n] = (-1, 3, -3, 1)
    D3[n - 1, n - 4:n] = (-1, 3, -3, 1)

    D4[0, 0:5] = (1, -4, 6, -4, 1)
    D4[1, 0:5] = (1, -4, 6, -4, 1)
    for i in range(2, n - 2):
        D4[i, i - 2:i + 3] = (1, -4, 6, -4, 1)
    D4[n - 2, n - 5:n] = (1, -4, 6, -4, 1)
    D4[n - 1, n - 5:n] = (1, -4, 6, -4, 1)

    C3[:] = np.eye(n)
    C3[0, 0] = 0; C3[1, 1] = 0
    C3[2, 2] = 163928591571.0 / 53268010936.0
    C3[3, 3] = 189284.0 / 185893.0
    C3[n - 5, n - 5] = C3[3, 3]
    C3[n - 4, n - 4] = 0
    C3[n - 3, n - 3] = C3[2, 2]
    C3[n - 2, n - 2] = 0
    C3[n - 1, n - 1] = 0

    C4[:] = np.eye(n)
    C4[0, 0] = 0; C4[1, 1] = 0
    C4[2, 2] = 1644330.0 / 301051.0
    C4[3, 3] = 156114.0 / 181507.0
    C4[n - 4, n - 4] = C4[3, 3]
    C4[n - 3, n - 3] = C4[2, 2]
    C4[n - 2, n - 2] = 0
    C4[n - 1, n - 1] = 0
    return D3, D4, C3, C4
