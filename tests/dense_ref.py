"""Independent dense (kron-product) restatement of the reference's gate and
observable definitions, used to pin the CPU oracle.

Matrices are the ones written in the reference's docstrings
(utils/cpu/cpuQuantumChannelGates.jl:53-71, :981-1100) and observables are
<psi|P|psi> with P built by kron products in the little-endian convention
(qubit k <-> bit k-1, utils/cpu/cpuQuantumStateObservables.jl:33-49).
"""
import numpy as np

I2 = np.eye(2, dtype=complex)
X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
Z = np.array([[1, 0], [0, -1]], dtype=complex)
H = np.array([[1, 1], [1, -1]], dtype=complex) / np.sqrt(2)
S = np.diag([1, 1j])
T = np.diag([1, np.exp(1j * np.pi / 4)])
SM = np.array([[0, 1], [0, 0]], dtype=complex)   # sigma- = |0><1|
SP = np.array([[0, 0], [1, 0]], dtype=complex)


def rx(t):
    c, s = np.cos(t / 2), np.sin(t / 2)
    return np.array([[c, -1j * s], [-1j * s, c]])


def ry(t):
    c, s = np.cos(t / 2), np.sin(t / 2)
    return np.array([[c, -s], [s, c]], dtype=complex)


def rz(t):
    return np.diag([np.exp(-1j * t / 2), np.exp(1j * t / 2)])


def embed(ops, N):
    """ops: {qubit(1-based): 2x2}; full 2^N operator, qubit N most significant."""
    M = np.array([[1]], dtype=complex)
    for q in range(N, 0, -1):
        M = np.kron(M, ops.get(q, I2))
    return M


def expm_herm(Hm, t):
    w, v = np.linalg.eigh(Hm)
    return (v * np.exp(-1j * w * t)) @ v.conj().T


def rpp(P, qi, qj, t, N):
    """exp(-i t/2 P_i P_j)"""
    PP = embed({qi: P, qj: P}, N)
    return expm_herm(PP, t / 2)


def controlled(U, c, t, N):
    P0 = np.diag([1, 0]).astype(complex)
    P1 = np.diag([0, 1]).astype(complex)
    return embed({c: P0}, N) + embed({c: P1, t: U}, N)


def ccz(a, b, c, N):
    dim = 1 << N
    d = np.ones(dim, dtype=complex)
    for i in range(dim):
        if (i >> (a - 1)) & 1 and (i >> (b - 1)) & 1 and (i >> (c - 1)) & 1:
            d[i] = -1
    return np.diag(d)


def toffoli(c1, c2, t, N):
    dim = 1 << N
    M = np.zeros((dim, dim), dtype=complex)
    for i in range(dim):
        j = i
        if (i >> (c1 - 1)) & 1 and (i >> (c2 - 1)) & 1:
            j = i ^ (1 << (t - 1))
        M[j, i] = 1
    return M


def two_qubit_local(U4, qa, qb, N):
    """U4 in the basis |00>,|qa=1>,|qb=1>,|11> (bit 0 = qa, bit 1 = qb)"""
    dim = 1 << N
    M = np.zeros((dim, dim), dtype=complex)
    for i in range(dim):
        a, b = (i >> (qa - 1)) & 1, (i >> (qb - 1)) & 1
        base = i & ~((1 << (qa - 1)) | (1 << (qb - 1)))
        col = a + 2 * b
        for r in range(4):
            j = base | ((r & 1) << (qa - 1)) | ((r >> 1) << (qb - 1))
            M[j, i] += U4[r, col]
    return M


def expect(psi, ops, N):
    P = embed(ops, N)
    return float(np.real(np.vdot(psi, P @ psi)))


def random_state(N, rng):
    v = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    return v / np.linalg.norm(v)
