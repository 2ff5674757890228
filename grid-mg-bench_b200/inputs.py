"""Seeded synthetic inputs for the multigrid hot path.

The reference draws its inputs from Grid's GridParallelRNG seeded with
{1,2,3,4} (e.g. src/Benchmark_create_coarse_operator.cc:108-113) and builds
gauge fields with SU3::HotConfiguration (:165).  Those streams cannot be
reproduced without Grid, so this module generates inputs with the same
distributions from numpy's PCG64 seeded with the same integers:

  gaussian_field   complex entries with re, im ~ N(0, 1/2)  (E|z|^2 = 1)
  hot_gauge        Haar-random SU(3) links (QR of a Gaussian matrix, phase-fixed)
  smooth_gauge     U = exp(i * eps * H), H a traceless Hermitian matrix with unit-variance
                   Gaussian entries (GUE: E|H_ij|^2 = 1), see gue_traceless
  random_links     Gaussian coarse link matrices, optionally with the
                   gamma5-hermiticity structure that ConstructRemainingLinks
                   produces (CoarsenedMatrixUpstreamImprovedDirsaveLut.h:1164-1196)

Layouts: gauge [site][mu][3][3], fields [site][rhs][dof], basis [i][site][dof],
links [point][site][N][N]; sites lexicographic with x fastest.
"""
import numpy as np

SEEDS = (1, 2, 3, 4)


def rng(seed=SEEDS, stream=0):
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence(list(seed) + [stream])))


def vol(dims):
    return int(np.prod(dims))


def gaussian_field(shape, r):
    a = r.standard_normal(tuple(shape) + (2,)) * np.sqrt(0.5)
    return (a[..., 0] + 1j * a[..., 1]).astype(np.complex128)


def _su3_project_phase(q):
    det = np.linalg.det(q)
    return q / (det ** (1.0 / 3.0))[..., None, None]


def hot_gauge(dims, r):
    """Haar-random SU(3) on every link."""
    n = vol(dims) * 4
    z = gaussian_field((n, 3, 3), r)
    q, rr = np.linalg.qr(z)
    d = np.diagonal(rr, axis1=-2, axis2=-1)
    q = q * (d / np.abs(d))[:, None, :]
    q = _su3_project_phase(q)
    return q.reshape(vol(dims), 4, 3, 3)


def gue_traceless(a):
    """Traceless Hermitian matrices with unit-variance Gaussian entries from complex
    unit-Gaussian matrices a (E|a_ij|^2 = 1): H = (a + a^dag) / sqrt(2) - tr/3.

    Every entry of H before the trace removal has E|H_ij|^2 = 1 (the Gaussian
    unitary ensemble), the plain reading of "Gaussian entries".  With this
    normalisation the smooth gauge field of eps = 0.3 puts the critical mass of
    the Wilson-clover operator (c_sw = 1, 32^4) near -0.39, so the multigrid
    configurations' masses (-0.3, -0.35) are near-critical but subcritical; the
    (a + a^dag) / 2 normalisation (variance 1/2) moves it to about -0.21, past
    which those masses lie.
    """
    import numpy as _np
    if isinstance(a, _np.ndarray):
        h = (a + _np.conj(_np.swapaxes(a, -1, -2))) / _np.sqrt(2.0)
        tr = _np.trace(h, axis1=-2, axis2=-1) / 3.0
        return h - tr[..., None, None] * _np.eye(3)
    import torch
    h = (a + a.conj().transpose(-1, -2)) / np.sqrt(2.0)
    tr = torch.diagonal(h, dim1=-2, dim2=-1).sum(-1) / 3.0
    return h - tr[..., None, None] * torch.eye(3, dtype=h.dtype, device=h.device)


def smooth_gauge(dims, r, eps):
    """U = exp(i eps H), H traceless Hermitian with unit-variance Gaussian entries."""
    n = vol(dims) * 4
    h = gue_traceless(gaussian_field((n, 3, 3), r))
    w, v = np.linalg.eigh(h)
    u = (v * np.exp(1j * eps * w)[:, None, :]) @ np.conj(np.swapaxes(v, -1, -2))
    return u.reshape(vol(dims), 4, 3, 3)


def shift_index(dims):
    """nbr[p][s] for the 9-point stencil (p<4: +dir p, 4<=p<8: -dir p-4, 8: self)."""
    V = vol(dims)
    s = np.arange(V)
    coords = []
    t = s.copy()
    for d in range(4):
        coords.append(t % dims[d])
        t //= dims[d]
    out = np.zeros((9, V), dtype=np.int64)
    for p in range(9):
        c = [x.copy() for x in coords]
        if p < 8:
            d = p % 4
            disp = 1 if p < 4 else -1
            c[d] = (c[d] + disp) % dims[d]
        idx = c[3]
        for d in (2, 1, 0):
            idx = idx * dims[d] + c[d]
        out[p] = idx
    return out


def random_links(dims, N, r, scale=None, g5_structure=True, diag_shift=0.0):
    """Gaussian coarse links [9][V][N][N].

    With g5_structure the forward links are rebuilt from the backward ones as
    A_{+mu}(x) = S o A_{-mu}(x+mu)^dag, S_{ab} = -1 iff a, b lie in different
    chiral halves, which is what a Galerkin coarsening of a gamma5-hermitian
    operator produces.  `scale` defaults to 1/sqrt(9 N) so that M keeps the
    norm of its input.  `diag_shift` adds a multiple of the identity to the
    self link.
    """
    V = vol(dims)
    if scale is None:
        scale = 1.0 / np.sqrt(9.0 * N)
    A = gaussian_field((9, V, N, N), r) * scale
    if g5_structure:
        nbr = shift_index(dims)
        half = N // 2
        k = np.arange(N) // half
        S = np.where((k[:, None] + k[None, :]) % 2 == 1, -1.0, 1.0)
        for d in range(4):
            back = A[4 + d]
            A[d] = S[None] * np.conj(np.swapaxes(back[nbr[d]], -1, -2))
        # self link: S o A_8 = A_8^dag
        A[8] = 0.5 * (A[8] + S[None] * np.conj(np.swapaxes(A[8], -1, -2)))
    if diag_shift:
        A[8] += diag_shift * np.eye(N)[None]
    return A


# ----------------------------------------------------------------------------
# Device-side generators for the large (32^4) configurations, seeded per stream.
# Same distributions as above, drawn with torch's Philox generator on the GPU.
# ----------------------------------------------------------------------------
def torch_gaussian(shape, seed, device="cuda", dtype=None):
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    re = torch.randn(tuple(shape), generator=g, device=device, dtype=torch.float64)
    im = torch.randn(tuple(shape), generator=g, device=device, dtype=torch.float64)
    z = torch.complex(re, im) * (0.5 ** 0.5)
    return z if dtype is None else z.to(dtype)


def torch_smooth_gauge(dims, seed, eps, device="cuda"):
    """U = exp(i eps H) per link, H traceless Hermitian with Gaussian entries -> [V][4][3][3] complex128."""
    import torch

    n = vol(dims) * 4
    h = gue_traceless(torch_gaussian((n, 3, 3), seed, device))
    # exp(i eps H) by scaling and squaring: Taylor series of exp(i eps H / 2^s) to
    # 18 terms (truncation below 1e-17 for |eps H / 2^s| <= 1/2), then s squarings
    a = (1j * eps) * h
    nrm = torch.linalg.matrix_norm(a, ord="fro").max().item()
    s = max(0, int(np.ceil(np.log2(max(nrm, 1e-30) / 0.5))))
    a = a / (2.0 ** s)
    eye = torch.eye(3, dtype=a.dtype, device=device).expand_as(a)
    u = eye.clone()
    term = eye.clone()
    for k in range(1, 19):
        term = term @ a / k
        u = u + term
    for _ in range(s):
        u = u @ u
    return u.reshape(vol(dims), 4, 3, 3).contiguous()
