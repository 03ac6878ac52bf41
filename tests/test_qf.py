"""Host side of the tensor-core mixed kernel (quadratic form, codegen/qf.py):
the basis covers the polynomial, the quadratic form is the polynomial, the
library's operand image is the restatement's byte for byte, and the kernel's
arithmetic (emulated in numpy) keeps the mixed-precision budget.  CPU only."""
import numpy as np
import pytest

from mbx_b200 import capi
from mbx_b200.codegen import qf, shift
from mbx_b200.codegen.gen_kernels import shifted_pip
from mbx_b200.specs import SPECS
from mbx_b200.tables import load_fit


@pytest.fixture(scope="module")
def mbpol3b():
    sp = shifted_pip("mbpol3b")
    return sp, qf.QuadForm("mbpol3b", sp)


@pytest.fixture(scope="module")
def liquid(mbpol3b):
    sp, _ = mbpol3b
    spec = SPECS["mbpol3b"]
    x = shift._variables(spec, shift.liquid_trimers(spec))
    return (x - sp.x0).astype(np.float32)


def test_basis_covers_every_monomial(mbpol3b):
    sp, q = mbpol3b
    assert q.nb <= q.npad == 480
    assert len(q.ij) == len(sp.monos)
    basis = set(q.basis)
    for (i, j), m in zip(q.ij, sp.monos):
        # the entry's two members multiply to the monomial
        assert tuple(sorted(q.basis[i] + q.basis[j])) == tuple(m)
        assert q.basis[i] in basis and q.basis[j] in basis
    # every member has degree <= 2 and appears once
    assert all(len(b) <= 2 for b in q.basis) and len(set(q.basis)) == q.nb


def test_quadratic_form_is_the_polynomial(mbpol3b):
    sp, q = mbpol3b
    rng = np.random.default_rng(5)
    a = load_fit("mbpol3b") * rng.uniform(0.5, 1.5, SPECS["mbpol3b"].ncoef)
    b0, b = shift.shifted_coefficients(sp, a)
    d = rng.uniform(-0.5, 0.5, (64, 36))
    direct = np.zeros(len(d))
    for m, o in zip(sp.monos, sp.orbit_of):
        if m:
            direct += b[o] * np.prod(d[:, list(m)], axis=1)
    M = np.zeros((len(d), q.npad))
    for j, bb in enumerate(q.basis):
        M[:, j] = np.prod(d[:, list(bb)], axis=1) if bb else 1.0
    qform = np.einsum("nj,jk,nk->n", M, q.matrix(b), M)
    np.testing.assert_allclose(qform, direct, rtol=0, atol=1e-11 * np.abs(direct).max())


@pytest.mark.parametrize("kind", ["fitted", "random"])
def test_library_image_matches_restatement(mbpol3b, kind):
    sp, q = mbpol3b
    a = load_fit("mbpol3b")
    if kind == "random":
        a = a * np.random.default_rng(11).normal(size=len(a))
    img, colf, b0 = capi.qf_image("mbpol3b", a)
    b0_ref, b = shift.shifted_coefficients(sp, a)
    img_ref, colf_ref = qf.image(q, b)
    assert img == img_ref
    np.testing.assert_array_equal(colf, colf_ref)
    assert b0 == b0_ref
    # nothing overflows the FP16 range, and the column factors are powers of two
    h = np.frombuffer(img, np.uint16)
    assert ((h & 0x7C00) != 0x7C00).all()
    assert (np.frexp(colf)[0] == 0.5).all()


def test_library_image_refuses_other_evaluators():
    with pytest.raises(RuntimeError):
        capi.qf_image("mbpol2b")


def test_emulated_kernel_precision(mbpol3b, liquid):
    """The kernel's arithmetic (FP16 splits, main and correction FP32
    accumulators rounded after every MMA) on 16,826 liquid trimers: summed
    energy within 1.5e-3 kcal/mol of the FP64 polynomial (5.9e-4; FP32
    products summed in FP64, as in the paired trie, are 2.4e-3 off here),
    every trimer within 1e-4, every variable gradient within 2e-3."""
    sp, q = mbpol3b
    b0, b = shift.shifted_coefficients(sp, load_fit("mbpol3b"))
    d = liquid.astype(np.float64)
    P_ref = np.zeros(len(d))
    g_ref = np.zeros(d.shape)
    for m, o in zip(sp.monos, sp.orbit_of):
        if not m:
            continue
        P_ref += b[o] * np.prod(d[:, list(m)], axis=1)
        for k, v in enumerate(m):
            rest = list(m[:k]) + list(m[k + 1:])
            g_ref[:, v] += b[o] * (np.prod(d[:, rest], axis=1) if rest else 1.0)
    P, g = q.emulate(b, liquid)
    assert abs(P.sum() - P_ref.sum()) < 1.5e-3
    assert np.abs(P - P_ref).max() < 1e-4
    assert np.abs(g - g_ref).max() < 2e-3


def test_row_scale_keeps_fp16_range(mbpol3b):
    _, q = mbpol3b
    rng = np.random.default_rng(2)
    d = (rng.normal(size=(256, 36)) * np.logspace(-3, 2.2, 256)[:, None]).astype(np.float32)
    r = q.row_scale(d)
    M = qf.monomial_values(q.basis, d).astype(np.float64)
    A = M * (2.0 ** -q.t[:q.nb])[None, :] * r[:, None]
    assert np.abs(A).max() < 2.0 ** 14
    assert (np.frexp(r)[0] == 0.5).all()
