"""GPU tests of the Gram step G = A^H A of kl_topk_eig (kl_factor_gram): the
integer-digit split on the tcgen05 tensor cores (S <= 256) and the FP64
CUDA-core GEMM beyond, against numpy's FP64 product of the same FP32 factor.

Tolerances: bit-exact where every entry of A is a multiple of 2^-12 of at
most 2^12 units (the digit split represents it exactly and every partial sum
is an FP64 integer); for a TCC factor (entries of one column share a
magnitude) max |G - G_fp64| <= 1e-9 max |G_fp64|; for columns of wide dynamic
range, the rounding bound of the split (2^-27 of each column's scale).
"""
import numpy as np
import pytest

import klitho as K
import synth

pytestmark = pytest.mark.gpu


def gram(A):
    import torch
    N, S = A.shape
    Ad = torch.from_numpy(np.ascontiguousarray(A, dtype=np.complex64)).cuda()
    G = torch.full((S, S), complex("nan"), dtype=torch.complex128, device="cuda")
    K.factor_gram(Ad, G)
    return G.cpu().numpy()


def ref(A):
    A64 = A.astype(np.complex128)
    return A64.conj().T @ A64


@pytest.mark.parametrize("N,S", [(1, 1), (100, 17), (1000, 64), (4099, 196), (2048, 256), (300, 300)])
def test_gram_exact_on_representable_factors(cuda, N, S):
    rng = np.random.default_rng(N + S)
    A = (rng.integers(-4096, 4097, (N, S)) + 1j * rng.integers(-4096, 4097, (N, S))) / 4096.0
    A[:, S // 2] *= 2.0 ** -30  # a column far below the others
    A = A.astype(np.complex64)
    G = gram(A)
    assert np.array_equal(G, ref(A))


def test_gram_tcc_factor_config4(cuda):
    import torch
    src = K.createSource(81, "CrossQuadrupole", radius=0.12, offset=0.75)
    tp = K.TccPlan(src, 1.35, synth.defocus_arg(25.0), 4096, 4096, n_medium=synth.N_WATER)
    A = torch.view_as_complex(tp.factor()).cpu().numpy()
    tp.close()
    assert A.shape == (11449, 196)
    G, R = gram(A), ref(A)
    assert np.abs(G - R).max() <= 1e-9 * np.abs(R).max()
    assert np.allclose(G, G.conj().T, rtol=0, atol=1e-15 * np.abs(R).max())
    assert np.all(np.diag(G).imag == 0.0)


def test_gram_wide_dynamic_range(cuda):
    # columns spanning six decades: the split rounds every entry to 2^-27 of its
    # column's scale 2^E (2^E <= 2 max|column|), so |G - G_fp64| stays within
    # sum_f |d_fs| |a_fs'| + |a_fs| |d_fs'| + |d_fs| |d_fs'| with |d| <= sqrt(2) 2^(E-28)
    rng = np.random.default_rng(5)
    N, S = 3000, 40
    A = (rng.standard_normal((N, S)) + 1j * rng.standard_normal((N, S))) * np.exp(rng.uniform(-14, 0, (N, 1)))
    A = A.astype(np.complex64)
    G, R = gram(A), ref(A)
    A64 = np.abs(A.astype(np.complex128))
    cm = np.maximum(np.abs(A.real), np.abs(A.imag)).max(axis=0).astype(np.float64)
    d = np.sqrt(2.0) * 2.0 ** (np.floor(np.log2(cm)) + 1 - 28)
    l1 = A64.sum(axis=0)
    bound = d[:, None] * l1[None, :] + l1[:, None] * d[None, :] + N * d[:, None] * d[None, :]
    assert np.all(np.abs(G - R) <= 1.01 * bound + 1e-15 * np.abs(R).max())
    assert np.abs(G - R).max() > 0.0  # the small entries were rounded: this is the bound, not exactness
