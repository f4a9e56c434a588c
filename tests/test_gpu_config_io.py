"""Gauge configurations as the reference's text files
(ovl_save_configuration / ovl_load_configuration against IO::SaveConfiguration
and IO::LoadConfiguration, IO/SaveConfiguration.cpp:3-62 and
IO/LoadConfiguration.cpp:3-148, run in the reference build).

Two colours: the files the device context writes are byte for byte the
reference's, and files the reference wrote load into the same numbers as the
reference's own loader reads (both parse the decimal text with correct
rounding).  Three colours, which the reference build here does not compile:
the layout the reference's SU(3) MatrixToString prints (nine "re im" pairs),
a round trip to within the 15 printed digits, and a second save that repeats
the first byte for byte.  Malformed files are refused and leave the fields
as they were."""
import numpy as np
import pytest

from _oracle import have_reference, ptr, reference
from overlap_b200 import Context, OvlError
from overlap_b200.inputs import random_efield, random_efield_su3, random_links, random_links_su3, volume

pytestmark = pytest.mark.gpu

N = (4, 3, 5)


def two_colour_fields(seed=11):
    return random_links(N, 0.7, seed), random_efield(N, 0.4, seed + 1)


def init_reference(U, E):
    R = reference("wilson")
    R.ovlref_init(*N, 1, 0, 0.05, 1.0, 0.0, 6.0, 0.05, 1.0, 7)
    R.ovlref_set_links(ptr(np.ascontiguousarray(U)))
    R.ovlref_set_efield(ptr(np.ascontiguousarray(E)))
    return R


@pytest.mark.skipif(not have_reference("wilson"), reason="reference build not present")
def test_saved_files_are_the_references_byte_for_byte(tmp_path):
    U, E = two_colour_fields()
    with Context(N=N, n_modes=32, precision="fp64") as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.save_configuration(tmp_path / "U.txt", tmp_path / "E.txt")
    R = init_reference(U, E)
    R.ovlref_save_configuration(str(tmp_path).encode(), 7, b"Uref", b"Eref")
    ours_u, ref_u = (tmp_path / "U.txt").read_bytes(), (tmp_path / "UrefID7.txt").read_bytes()
    ours_e, ref_e = (tmp_path / "E.txt").read_bytes(), (tmp_path / "ErefID7.txt").read_bytes()
    assert ours_u.count(b"\n") == 3 * volume(N) and ours_u == ref_u
    assert ours_e.count(b"\n") == 3 * volume(N) and ours_e == ref_e


@pytest.mark.skipif(not have_reference("wilson"), reason="reference build not present")
def test_reference_files_load_as_the_reference_loads_them(tmp_path):
    U, E = two_colour_fields(seed=21)
    R = init_reference(U, E)
    R.ovlref_save_configuration(str(tmp_path).encode(), 3, b"UOutT0", b"EOutT0")
    R.ovlref_set_links(ptr(np.zeros_like(U)))
    R.ovlref_load_configuration(str(tmp_path).encode(), b"UOutT0ID3.txt", b"EOutT0ID3.txt")
    ref_u, ref_e = np.zeros_like(U), np.zeros_like(E)
    R.ovlref_get_links(ptr(ref_u))
    R.ovlref_get_efield(ptr(ref_e))
    with Context(N=N, n_modes=32, precision="fp64") as ctx:
        ctx.load_configuration(tmp_path / "UOutT0ID3.txt", tmp_path / "EOutT0ID3.txt")
        got_u, got_e = ctx.get_links(), ctx.get_efield()
    assert np.array_equal(got_u, ref_u) and np.array_equal(got_e, ref_e)
    assert np.max(np.abs(got_u - U)) < 1e-14 and np.max(np.abs(got_e - E)) < 1e-14


def test_three_colour_files_follow_the_su3_layout_and_round_trip(tmp_path):
    U, E = random_links_su3(N, 0.6, 5), random_efield_su3(N, 0.3, 6)
    V = volume(N)
    with Context(N=N, n_colours=3, n_modes=32, precision="fp64") as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.save_configuration(tmp_path / "U.txt", tmp_path / "E.txt")
    lines = (tmp_path / "U.txt").read_text().splitlines()
    assert len(lines) == 3 * V and all(line.endswith(" ") for line in lines)
    rows = np.array([line.split() for line in lines], dtype=float)
    assert rows.shape == (3 * V, 4 + 18)
    # z outermost, then y, x, the direction innermost
    z, y, x, mu = np.meshgrid(np.arange(N[2]), np.arange(N[1]), np.arange(N[0]), np.arange(3), indexing="ij")
    assert np.array_equal(rows[:, :4].astype(int), np.stack([x, y, z, mu], -1).reshape(-1, 4))
    flat = np.ascontiguousarray(U).view(np.float64).reshape(V, 3, 18)  # [site][mu][re im x 9]
    assert np.max(np.abs(rows[:, 4:] - flat.reshape(-1, 18))) < 1e-14
    erows = np.array([line.split() for line in (tmp_path / "E.txt").read_text().splitlines()], dtype=float)
    assert erows.shape == (3 * V, 4 + 8) and np.max(np.abs(erows[:, 4:] - E.reshape(-1, 8))) < 1e-15
    with Context(N=N, n_colours=3, n_modes=32, precision="fp64") as ctx:
        ctx.load_configuration(tmp_path / "U.txt", tmp_path / "E.txt")
        assert np.max(np.abs(ctx.get_links() - U)) < 1e-14 and np.max(np.abs(ctx.get_efield() - E)) < 1e-15
        ctx.save_configuration(tmp_path / "U2.txt", tmp_path / "E2.txt")
    assert (tmp_path / "U2.txt").read_bytes() == (tmp_path / "U.txt").read_bytes()
    assert (tmp_path / "E2.txt").read_bytes() == (tmp_path / "E.txt").read_bytes()


def test_malformed_files_are_refused_and_leave_the_fields(tmp_path):
    U, E = two_colour_fields(seed=31)
    with Context(N=N, n_modes=32, precision="fp64") as ctx:
        ctx.set_links(U)
        ctx.set_efield(E)
        ctx.save_configuration(tmp_path / "U.txt", tmp_path / "E.txt")
        good = (tmp_path / "U.txt").read_text().splitlines(keepends=True)
        ctx.set_links(random_links(N, 0.2, 99))  # the state the failed loads must keep
        before = ctx.get_links()
        cases = {"missing": good[:-1], "twice": good[:-1] + good[:1], "outside": good[:-1] + ["9 0 0 0 1 0 0 0 \n"],
                 "short": good[:-1] + [" ".join(good[-1].split()[:6]) + "\n"]}
        for name, text in cases.items():
            path = tmp_path / f"bad_{name}.txt"
            path.write_text("".join(text))
            with pytest.raises(OvlError, match=f"bad_{name}"):
                ctx.load_configuration(path, tmp_path / "E.txt")
            assert np.array_equal(ctx.get_links(), before), name
        with pytest.raises(OvlError, match="cannot open"):
            ctx.load_configuration(tmp_path / "absent.txt", None)
        # blank lines and any line order are accepted
        path = tmp_path / "shuffled.txt"
        path.write_text("\n" + "".join(good[::-1]) + "\n\n")
        ctx.load_configuration(path, None)
        assert np.max(np.abs(ctx.get_links() - U)) < 1e-14
