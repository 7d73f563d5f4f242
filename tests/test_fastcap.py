"""FastCap decks (.qui panel files and .lst conductor lists) in front of the
field solver.

CPU: the reader follows the reference's parser (cap/geometry.rs:55-135,
cap/listfile.rs:42-115): line kinds, conductor numbering and naming, scaling,
translation, and the error messages with their line numbers.
GPU: a parsed deck solved through gpx_cap_solve equals the oracle's dense
LU solve (cap::solve, Method::Direct) of the same panels to 1e-9, for
quadrilateral and triangular panels; a list file's permittivity scales the
matrix, and a list of several permittivities (gpx_cap_solve_eps) equals the
oracle's restatement of cap/dielectric.rs:76-150 with conductor roles."""
import numpy as np
import pytest

from gpurify_b200 import fastcap
from tests.helpers import rel_max


def plate_qui(num, x0, y0, z, lx, ly, nx, ny, triangles=False):
    """A rectangular plate as FastCap panel lines for conductor `num`."""
    out = []
    dx, dy = lx / nx, ly / ny
    for i in range(nx):
        for j in range(ny):
            a = (x0 + i * dx, y0 + j * dy, z)
            b = (x0 + (i + 1) * dx, y0 + j * dy, z)
            c = (x0 + (i + 1) * dx, y0 + (j + 1) * dy, z)
            d = (x0 + i * dx, y0 + (j + 1) * dy, z)
            if triangles:
                out.append("T %d " % num + " ".join("%.17g" % t for p in (a, b, c) for t in p))
                out.append("T %d " % num + " ".join("%.17g" % t for p in (a, c, d) for t in p))
            else:
                out.append("Q %d " % num + " ".join("%.17g" % t for p in (a, b, c, d) for t in p))
    return "\n".join(out) + "\n"


def test_qui_line_kinds_numbering_and_names():
    text = ("0 title line of the deck\n"
            "* a comment\n"
            "% another comment\n"
            "\n"
            "N 7 top\n"
            "Q 7 0 0 1  2 0 1  2 3 1  0 3 1\n"
            "t 3 0 0 0  1 0 0  0 1 0  extra tokens ignored\n"
            "q 7 0 0 2  1 0 2  1 1 2  0 1 2\n"
            "n 3 bottom\n")
    g = fastcap.parse(text, scale=0.5)
    assert g.num_conductors() == 2
    assert g.conductor_names == ["top", "bottom"]
    assert g.numbers == [7, 3]
    assert g.cond.tolist() == [0, 1, 0]
    assert g.verts.shape == (3, 12)
    np.testing.assert_array_equal(g.verts[0], 0.5 * np.array([0, 0, 1, 2, 0, 1, 2, 3, 1, 0, 3, 1.0]))
    # a triangle repeats its third vertex
    np.testing.assert_array_equal(g.verts[1], 0.5 * np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 1, 0.0]))
    # unnamed conductors are called cond<number>
    assert fastcap.parse("Q 12 0 0 0 1 0 0 1 1 0 0 1 0\n").conductor_names == ["cond12"]


@pytest.mark.parametrize("text,msg", [
    ("0 t\nQ\n", "line 2: Q: missing conductor number"),
    ("T x 0 0 0 1 0 0 0 1 0\n", "line 1: T: missing conductor number"),
    ("Q 1 0 0 0 1 0 0 1 1 0\n", "line 1: expected 12 numbers, got 9"),
    ("\n\nT 1 0 0 0 1 0 0 0 1 zz\n", "line 3: bad number 'zz'"),
    ("C sub.qui\n", "line 1: C (sub-file include) not yet supported"),
    ("X 1 2 3\n", "line 1: unrecognized line: X 1 2 3"),
])
def test_qui_errors_name_the_line(text, msg):
    with pytest.raises(fastcap.FastCapError) as e:
        fastcap.parse(text)
    assert str(e.value) == msg


def test_list_file_translates_and_numbers_per_file(tmp_path):
    (tmp_path / "pair.qui").write_text(plate_qui(4, 0, 0, 0, 1, 1, 1, 1) + plate_qui(9, 0, 0, 0.5, 1, 1, 2, 1))
    (tmp_path / "one.qui").write_text(plate_qui(1, 0, 0, 0, 2, 2, 1, 1))
    lst = ("* deck\n"
           "C pair.qui 2.5 0 0 0\n"
           "% comment\n"
           "C one.qui 2.5 10 20 30 +\n"
           "c pair.qui 2.5 0 0 5\n")
    (tmp_path / "deck.lst").write_text(lst)
    g = fastcap.parse_list_file(str(tmp_path / "deck.lst"))
    assert g.conductor_names == ["pair.qui:0", "pair.qui:1", "one.qui:0", "pair.qui:0", "pair.qui:1"]
    assert g.num_conductors() == 5 and len(g.verts) == 3 + 1 + 3
    assert g.cond.tolist() == [0, 1, 1, 2, 3, 4, 4]
    assert g.eps_r == 2.5
    np.testing.assert_allclose(g.verts[3].reshape(4, 3), np.array([[10, 20, 30], [12, 20, 30], [12, 22, 30],
                                                                   [10, 22, 30.0]]))
    np.testing.assert_allclose(g.verts[4].reshape(4, 3)[:, 2], 5.0)


@pytest.mark.parametrize("lst,msg", [
    ("D a.qui 1 3.9 0 0 0 0 0 0\n", "line 1: dielectric interfaces"),
    ("C\n", "line 1: C: missing file"),
    ("C a.qui 1 0 zero 0\n", "line 1: expected number for ytrans"),
    ("L a.qui\n", "line 1: unrecognized list line: L a.qui"),
    ("C missing.qui 1 0 0 0\n", "cannot read"),
    ("* x\nC bad.qui 1 0 0 0\n", "geometry parse error in 'bad.qui': line 1: Q: missing conductor number "
                                 "(line 2 of list)"),
])
def test_list_errors(tmp_path, lst, msg):
    (tmp_path / "a.qui").write_text(plate_qui(1, 0, 0, 0, 1, 1, 1, 1))
    (tmp_path / "bad.qui").write_text("Q\n")
    with pytest.raises(fastcap.FastCapError) as e:
        fastcap.parse_list_str(lst, str(tmp_path))
    assert msg in str(e.value)


def test_list_with_several_permittivities_keeps_them_per_panel(tmp_path):
    (tmp_path / "a.qui").write_text(plate_qui(1, 0, 0, 0, 1, 1, 2, 1))
    (tmp_path / "b.qui").write_text(plate_qui(1, 0, 0, 0, 1, 1, 1, 3))
    g = fastcap.parse_list_str("C a.qui 3.9 0 0 0\nC b.qui 2.5 0 0 1\nC a.qui 3.9 0 0 2\n", str(tmp_path))
    assert g.panel_eps.tolist() == [3.9, 3.9, 2.5, 2.5, 2.5, 3.9, 3.9]
    assert len(g.panel_eps) == len(g.verts)
    one = fastcap.parse_list_str("C a.qui 3.9 0 0 0\nC b.qui 3.9 0 0 1\n", str(tmp_path))
    assert one.panel_eps is None and one.eps_r == 3.9


@pytest.fixture(scope="module")
def ctx():
    from gpurify_b200 import _lib

    c = _lib.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("triangles", [False, True])
def test_qui_deck_solves_like_the_oracle_lu(ctx, orc, triangles):
    text = "0 two plates, 1 mm apart\n" + plate_qui(1, 0, 0, 0, 0.02, 0.03, 8, 10, triangles) + \
        plate_qui(2, 0.001, -0.002, 0.001, 0.018, 0.034, 9, 11, triangles)
    g = fastcap.parse(text)
    C, rep = fastcap.solve(g, ctx)
    assert rep["dense"] == 1 and rep["converged"] == 1
    ref = orc.cap_dense(g.verts, g.cond, 2)
    assert rel_max(C, ref) < 1e-9
    # collocation leaves C slightly unsymmetric on unlike meshes (about 1e-3 here)
    assert C[0, 1] < 0 < C[0, 0] and abs(C[0, 1] - C[1, 0]) < 1e-2 * abs(C[0, 1])


@pytest.mark.gpu
def test_list_permittivity_scales_the_matrix(ctx, tmp_path):
    (tmp_path / "bot.qui").write_text(plate_qui(1, 0, 0, 0, 0.01, 0.01, 6, 6))
    (tmp_path / "top.qui").write_text(plate_qui(1, 0, 0, 0, 0.01, 0.01, 6, 6))
    vac = fastcap.parse_list_str("C bot.qui 1 0 0 0\nC top.qui 1 0 0 0.0005\n", str(tmp_path))
    die = fastcap.parse_list_str("C bot.qui 3.9 0 0 0\nC top.qui 3.9 0 0 0.0005\n", str(tmp_path))
    C1, _ = fastcap.solve(vac, ctx)
    C2, _ = fastcap.solve(die, ctx)
    np.testing.assert_allclose(C2, 3.9 * C1, rtol=1e-14)
    # parallel plates 1 cm square, 0.5 mm apart: eps0 A / d plus a few percent of fringing
    eps0 = 8.8541878128e-12
    assert 1.0 < -C1[0, 1] / (eps0 * 1e-4 / 5e-4) < 1.3


@pytest.mark.gpu
def test_list_with_several_permittivities_matches_the_oracle(ctx, orc, tmp_path):
    """cap/dielectric.rs:76-150 with conductor roles: each panel's charge
    counts with its own line's permittivity; all pairs, against the oracle's
    LU restatement to 1e-9."""
    (tmp_path / "bot.qui").write_text(plate_qui(1, 0, 0, 0, 0.01, 0.01, 6, 6))
    (tmp_path / "top.qui").write_text(plate_qui(1, 0, 0, 0, 0.01, 0.01, 5, 7))
    g = fastcap.parse_list_str("C bot.qui 3.9 0 0 0\nC top.qui 2.2 0 0 0.0005\n", str(tmp_path))
    C, rep = fastcap.solve(g, ctx)
    assert rep["dense"] == 1 and rep["converged"] == 1
    ref = orc.cap_dense_eps(g.verts, g.cond, 2, g.panel_eps)
    assert rel_max(C, ref) < 1e-9
    # one permittivity per conductor: row i is the vacuum row times conductor i's
    C1, _ = fastcap.solve(fastcap.parse_list_str("C bot.qui 1 0 0 0\nC top.qui 1 0 0 0.0005\n", str(tmp_path)),
                          ctx)
    np.testing.assert_allclose(C, np.array([[3.9], [2.2]]) * C1, rtol=1e-12)
