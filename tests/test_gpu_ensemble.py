"""Ensembles (ovl_ensemble_*): trajectories of mixed lattice sizes, mode counts
and physics stepped together by batched launches under a CUDA graph.  Each
member must evolve exactly as the same context stepped alone (the batched hop
runs the single-context stencil; separately compiled kernels may contract
multiply-adds differently, so the comparison allows the last bits), including a
U(1) background, reunitarisation and a tSphaleron gate crossed mid-run."""
import numpy as np
import pytest

from _helpers import random_modes, rel_err
from overlap_b200 import Context, Ensemble, OvlError, Params
from overlap_b200.inputs import random_efield, random_links

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(N=(4, 5, 6), n_modes=70, first_mode=1, m_fermion=0.1, dt=0.05, t_sphaleron=1e9),
    dict(N=(6, 6, 6), n_modes=33, first_mode=0, m_fermion=0.05, dt=0.04, t_sphaleron=0.1, reunitarize=True),
    dict(N=(5, 4, 4), n_modes=64, first_mode=2, m_fermion=0.2, dt=0.05, t_sphaleron=1e9),
    dict(N=(5, 5, 3), n_modes=45, first_mode=0, m_fermion=0.1, dt=0.05, t_sphaleron=1e9),  # V = 75: a partial tile
]


def inputs(i, kw):
    N = kw["N"]
    n = kw["n_modes"]
    return (random_links(N, 0.5, 10 * i + 1), random_efield(N, 0.3, 10 * i + 2), random_modes(n, N, 10 * i + 3),
            random_modes(n, N, 10 * i + 4))


def phases(N, seed):
    return np.exp(1j * np.random.default_rng(seed).uniform(-np.pi, np.pi, (N[1], N[0], 2)))


def solo_variant(precision, tile):
    """The single-context hop variant with the arithmetic of the ensemble's tiles."""
    return 3 if tile == 16 and precision == "fp32" else 0


@pytest.mark.parametrize("precision,tile", [("fp32", 0), ("fp64", 0), ("fp32", 16), ("fp64", 16)])
def test_ensemble_members_evolve_as_alone(precision, tile):
    """tile 0: the tile shape is tuned; 16: packed-pair tiles for the FP32
    members (FP64 members fall back to tiles of 8 sites); V = 120, 216, 80 and
    2-3 mode blocks leave partial tiles."""
    params = [Params(precision=precision, form="fused", m_dw=0.0, hop_variant=solo_variant(precision, tile), **kw)
              for kw in MEMBERS]
    alone = []
    for i, (p, kw) in enumerate(zip(params, MEMBERS)):
        U, E, psi0, mid0 = inputs(i, kw)
        with Context(p) as ctx:
            ctx.set_links(U)
            ctx.set_efield(E)
            if i == 2:
                ctx.set_u1(phases(kw["N"], 5))
            ctx.set_modes(psi0, mid0)
            ctx.step(5)
            alone.append((ctx.get_modes(), ctx.get_links(), ctx.charges()))
    with Ensemble(params) as ens:
        if tile:
            ens.set_tile(tile)
        for i, kw in enumerate(MEMBERS):
            U, E, psi0, mid0 = inputs(i, kw)
            ens[i].set_links(U)
            ens[i].set_efield(E)
            if i == 2:
                ens[i].set_u1(phases(kw["N"], 5))
            ens[i].set_modes(psi0, mid0)
        ens.step(2)
        ens.step(3)  # the step graph is replayed with re-uploaded descriptors
        ch = ens.charges()
        info = ens.info()
        tol = 1e-13 if precision == "fp64" else 1e-5
        for i in range(len(MEMBERS)):
            (psi, mid), U, c = alone[i]
            bpsi, bmid = ens[i].get_modes()
            assert rel_err(bpsi, psi) < tol and rel_err(bmid, mid) < tol, i
            assert rel_err(ens[i].get_links(), U) < 1e-14, i
            assert ens[i].step_count == 5
            for k, name in enumerate(("NV", "N5", "PS", "WA")):
                assert abs(ch[i, k] - c[name]) <= tol * max(1.0, abs(c[name])), (i, name)
    assert info["sites"] == tile if tile else info["sites"] in ((4, 8, 16) if precision == "fp32" else (4, 8))
    assert info["launches"] >= 25


def test_tile_shape_change_between_steps():
    """Changing the tile shape between steps (ovl_ensemble_set_tile drops the
    captured step graph; a single member's descriptor is the same for every
    shape) keeps the evolution right: 3 steps with 8-site tiles, then 3 with
    packed tiles, agree with the member stepped alone with hop variant 0 and
    then 3 to FP32 rounding, and the ensemble reports the shape set.  (Both tile
    kernels compute the same operator, so this checks the results, not which
    kernel ran.)"""
    kw = dict(N=(4, 5, 6), n_modes=70, first_mode=1, m_fermion=0.1, dt=0.05, t_sphaleron=1e9)
    U, E, psi0, mid0 = inputs(0, kw)
    p0 = Params(precision="fp32", form="fused", m_dw=0.0, hop_variant=0, **kw)
    with Context(p0) as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.set_modes(psi0, mid0)
        ctx.step(3)
        psi3, mid3 = ctx.get_modes()
        U3, E3 = ctx.get_links(), ctx.get_efield()
    with Context(Params(precision="fp32", form="fused", m_dw=0.0, hop_variant=3, **kw)) as ctx:
        ctx.set_links(U3)
        ctx.set_efield(E3)
        ctx.set_modes(psi3, mid3)
        ctx.step(3)
        alone = ctx.get_modes()
    with Ensemble([p0]) as ens:
        ens.set_tile(8)
        ens[0].set_links(U)
        ens[0].set_efield(E)
        ens[0].set_modes(psi0, mid0)
        ens.step(3)
        assert ens.info()["sites"] == 8
        ens.set_tile(16)
        ens.step(3)
        assert ens.info()["sites"] == 16
        got = ens[0].get_modes()
    assert rel_err(got[0], alone[0]) < 1e-5 and rel_err(got[1], alone[1]) < 1e-5


def test_packed_tiles_beyond_one_cta_row_of_mode_blocks():
    """Packed-pair tiles run 8 mode blocks per CTA; a member of 300 modes (10
    blocks, the last one 12 of 32 lanes) needs a second row of them (mbt > 0 in
    wilson_batch_packed_kernel), beside a member of 70 modes, one with a U(1)
    background: each member as alone with hop variant 3."""
    kws = [dict(N=(4, 5, 6), n_modes=300, first_mode=1, m_fermion=0.1, dt=0.05, t_sphaleron=1e9),
           dict(N=(4, 5, 6), n_modes=70, first_mode=0, m_fermion=0.05, dt=0.05, t_sphaleron=0.1)]
    params = [Params(precision="fp32", form="fused", m_dw=0.0, hop_variant=3, **kw) for kw in kws]
    alone = []
    for i, (p, kw) in enumerate(zip(params, kws)):
        U, E, psi0, mid0 = inputs(i, kw)
        with Context(p) as ctx:
            ctx.set_links(U)
            ctx.set_efield(E)
            if i == 0:
                ctx.set_u1(phases(kw["N"], 8))
            ctx.set_modes(psi0, mid0)
            ctx.step(4)
            alone.append((ctx.get_modes(), ctx.charges()))
    with Ensemble(params) as ens:
        ens.set_tile(16)
        for i, kw in enumerate(kws):
            U, E, psi0, mid0 = inputs(i, kw)
            ens[i].set_links(U)
            ens[i].set_efield(E)
            if i == 0:
                ens[i].set_u1(phases(kw["N"], 8))
            ens[i].set_modes(psi0, mid0)
        ens.step(4)
        ch = ens.charges()
        for i in range(len(kws)):
            (psi, mid), c = alone[i]
            bpsi, bmid = ens[i].get_modes()
            assert rel_err(bpsi, psi) < 1e-5 and rel_err(bmid, mid) < 1e-5, i
            assert abs(ch[i, 1] - c["N5"]) <= 1e-5 * max(1.0, abs(c["N5"])), i


def test_ensemble_rejects_an_unknown_tile_shape():
    with Ensemble([Params(N=(4, 4, 4), n_modes=8, form="fused", precision="fp32")]) as ens:
        with pytest.raises(OvlError):
            ens.set_tile(5)
        ens.set_tile(16)
        ens.set_tile(0)


def test_ensemble_rejects_unsupported_members():
    with pytest.raises(OvlError):
        Ensemble([Params(N=(4, 4, 4), n_modes=8, form="plain")])
    with pytest.raises(OvlError):
        Ensemble([Params(N=(4, 4, 4), n_modes=8, form="fused", precision="fp32"),
                  Params(N=(4, 4, 4), n_modes=8, form="fused", precision="fp64")])


@pytest.mark.parametrize("precision,tile", [("fp32", 0), ("fp64", 0), ("fp32", 16)])
def test_three_colour_members_batch_beside_two_colour_ones(precision, tile):
    """SU(3) members (with and without a U(1) background) in the same ensemble
    as SU(2) ones: one batched launch per group, each member as alone (with
    packed tiles the SU(2) group runs packed, the SU(3) groups 8-site tiles)."""
    from overlap_b200.inputs import random_efield_su3, random_links_su3, volume

    def modes3(n, N, seed):
        rng = np.random.default_rng(seed)
        shape = (n, volume(N), 3, 4)
        return rng.normal(0, np.sqrt(0.5), shape) + 1j * rng.normal(0, np.sqrt(0.5), shape)

    kws = [dict(N=(4, 4, 6), n_modes=40, m_fermion=0.1, dt=0.05, t_sphaleron=1e9, n_colours=3),
           dict(N=(4, 5, 4), n_modes=64, m_fermion=0.05, dt=0.05, t_sphaleron=1e9, n_colours=3, reunitarize=True),
           dict(N=(6, 4, 4), n_modes=33, m_fermion=0.1, dt=0.05, t_sphaleron=1e9, n_colours=2)]
    params = [Params(precision=precision, form="fused", m_dw=0.0,
                     hop_variant=solo_variant(precision, tile) if kw["n_colours"] == 2 else 0, **kw) for kw in kws]

    def setup(ctx, i, kw):
        N = kw["N"]
        if kw["n_colours"] == 3:
            ctx.set_links(random_links_su3(N, 0.6, 50 + i))
            ctx.set_efield(random_efield_su3(N, 0.3, 60 + i))
            ctx.set_modes(modes3(kw["n_modes"], N, 70 + i), modes3(kw["n_modes"], N, 80 + i))
        else:
            ctx.set_links(random_links(N, 0.6, 50 + i))
            ctx.set_efield(random_efield(N, 0.3, 60 + i))
            ctx.set_modes(random_modes(kw["n_modes"], N, 70 + i), random_modes(kw["n_modes"], N, 80 + i))
        if i == 1:
            ctx.set_u1(phases(N, 9))

    alone = []
    for i, (p, kw) in enumerate(zip(params, kws)):
        with Context(p) as ctx:
            setup(ctx, i, kw)
            ctx.step(4)
            alone.append((ctx.get_modes()[0], ctx.get_links(), ctx.charges()["N5"]))
    with Ensemble(params) as ens:
        if tile:
            ens.set_tile(tile)
        for i, kw in enumerate(kws):
            setup(ens[i], i, kw)
        ens.step(4)
        n5 = ens.charges()[:, 1]
        tol = 1e-13 if precision == "fp64" else 1e-5
        for i in range(len(kws)):
            psi, U, c = alone[i]
            assert rel_err(ens[i].get_modes()[0], psi) < tol, i
            assert rel_err(ens[i].get_links(), U) < 1e-13, i
            assert abs(n5[i] - c) <= tol * max(1.0, abs(c)), i
        # groups: SU(2) plain, SU(3) plain, SU(3) with U(1): 3 hop launches per half step + 3
        assert ens.info()["launches"] >= 4 * 9
