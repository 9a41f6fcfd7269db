"""CPU tests of the input-deck reader and the reference-deck problem setup."""
import dataclasses
import pathlib

import numpy as np
import pytest

from oracle.bindings import RefSnap
from snap_b200 import input_deck as D
from snap_b200 import problem as P

DECKS = pathlib.Path(__file__).resolve().parent / "decks"
ALL = sorted(DECKS.glob("*.in"))


def test_every_reference_deck_parses():
    assert len(ALL) == 24
    for f in ALL:
        df = D.parse_deck(f)
        d = df.deck
        assert d.cells == df.values["nx"] * df.values["ny"] * df.values["nz"]
        assert d.timedep == bool(df.values["timedep"])


def test_deck_values():
    d = D.parse_deck(DECKS / "huge_4K_1x1x1.in").deck
    assert (d.nx, d.ny, d.nz, d.nang, d.ng, d.nmom) == (16, 16, 16, 1024, 96, 1)
    assert d.timedep and d.nsteps == 10 and d.tf == 10.0 and d.dt == 1.0
    assert d.lx == 0.6 and d.epsi == 1e-4 and (d.iitm, d.oitm) == (5, 100)
    assert d.mat_opt == 0 and d.src_opt == 0 and d.nmat == 1
    t = D.parse_deck(DECKS / "test.in").deck
    assert t.chunks == (2, 2, 2) and not t.timedep
    assert D.parse_deck(DECKS / "mms.in").deck.src_opt == 3


def test_grid_factors_follow_the_reference():
    d = D.parse_deck(DECKS / "small_4K_1x1x1.in").deck
    assert d.h == (2.0 / (0.6 / 16),) * 3        # snap.cc:1178-1180


def _text(**over):
    base = (DECKS / "simple.in").read_text()
    for k, v in over.items():
        base = base.replace(f"  {k}=", f"  {k}=XX", 1)
        lines = base.splitlines()
        base = "\n".join(f"  {k}={v}" if ln.strip().startswith(f"{k}=XX") else ln for ln in lines)
    return base


@pytest.mark.parametrize("bad,msg", [({"angcpy": 1}, "angcpy"), ({"swp_typ": 0}, "swp_typ"),
                                     ({"nmom": 5}, "nmom"), ({"ndimen": 2}, "ndimen"),
                                     ({"npey": 3}, "ny % npey"), ({"mat_opt": 4}, "mat_opt")])
def test_invalid_decks_are_rejected(bad, msg):
    with pytest.raises(ValueError, match=msg):
        D.parse_deck_text(_text(**bad))


def test_entries_must_come_in_order():
    text = (DECKS / "simple.in").read_text().replace("  nx=32\n  lx=0.6\n", "  lx=0.6\n  nx=32\n")
    with pytest.raises(ValueError, match="expected 'nx='"):
        D.parse_deck_text(text)


def test_report_arguments(capsys):
    D.report_arguments(D.parse_deck(DECKS / "mms.in"))
    out = capsys.readouterr().out
    assert "Source Layout: MMS" in out and "X-Chunks: 2" in out and "Angles: 16" in out


@pytest.mark.skipif(not RefSnap.available(), reason="reference build not present")
@pytest.mark.parametrize("mat_opt,src_opt", [(0, 0), (1, 1), (2, 2), (1, 2), (2, 0)])
def test_layouts_match_reference_init(mat_opt, src_opt):
    """reference_layout against the reference's own InitMaterial /
    InitSource tasks (init.cc:49-191) on an uneven mesh."""
    d = P.Deck(12, 10, 6, nang=4, ng=3, nmom=1, mat_opt=mat_opt, src_opt=src_opt)
    mat, qi = RefSnap(d).init_layout()
    pm, pq = P.reference_layout(d)
    assert np.array_equal(mat, pm)
    assert np.array_equal(qi, pq)


def test_reference_cross_sections():
    """Spot values of Snap::initialize_scattering (snap.cc:571-714), G = 3."""
    sigt, slgg = P.reference_cross_sections(3, 2, True)
    assert np.allclose(sigt[:, 0], [1.0, 0.01, 1e-4]) and np.allclose(sigt[:, 1], [2.0, 0.02, 2e-4])
    sigs1 = np.array([0.5, 0.0025, 0.0000125])
    # source group 0, material 1: 0.3 in-group, 0.7 split over groups 1 and 2
    assert np.isclose(slgg[0, 0, 0, 0], 0.3 * sigs1[0])
    assert np.isclose(slgg[1, 0, 0, 0], 0.35 * sigs1[0]) and np.isclose(slgg[2, 0, 0, 0], 0.35 * sigs1[0])
    # source group 1: 0.2 in-group, 0.1 up to group 0, 0.7 down to group 2
    assert np.isclose(slgg[1, 0, 1, 0], 0.2 * sigs1[1])
    assert np.isclose(slgg[0, 0, 1, 0], 0.1 * sigs1[1]) and np.isclose(slgg[2, 0, 1, 0], 0.7 * sigs1[1])
    # last group keeps 0.9 in-group, 0.1 split over the two above
    assert np.isclose(slgg[2, 0, 2, 0], 0.9 * sigs1[2]) and np.isclose(slgg[0, 0, 2, 0], 0.05 * sigs1[2])
    # material 2: 0.6 first group in-group, Legendre order 1 scaled by 0.8
    assert np.isclose(slgg[0, 1, 0, 0], 0.6 * 1.2) and np.isclose(slgg[0, 1, 0, 1], 0.8 * 0.6 * 1.2)
    assert np.isclose(slgg[0, 0, 0, 1], 0.1 * slgg[0, 0, 0, 0])
    one, s1 = P.reference_cross_sections(1, 1, False)
    assert s1.shape == (1, 1, 1, 1) and s1[0, 0, 0, 0] == 0.5


@pytest.mark.skipif(not RefSnap.available(), reason="reference build not present")
def test_reference_time_dependent_solve_runs():
    """The reference's own task bodies step a time-dependent deck (the
    GPU tests compare against this)."""
    d = D.parse_deck(DECKS / "tiny_512_1x1x1.in").deck
    flux, rec = RefSnap(d).solve(P.make_problem(d), nthreads=2)
    assert rec["outer_total"] >= d.nsteps and np.all(np.isfinite(flux)) and flux.min() > 0


@pytest.mark.skipif(not RefSnap.available(), reason="reference build not present")
def test_reference_chunked_run_matches_one_chunk():
    """The reference run of a 2x2x2-chunk deck sweeps each chunk as its own
    task, upstream chunks first, faces passed through the shared face arrays
    (snap.cc:56-62, 849-887); the flux and iteration record equal those of
    the same deck in one chunk to rounding, which is why the GPU sweeps the
    whole mesh as one domain.  The MMS deck's tasks also run per chunk; its
    comparison sum is the same, its average divided by the chunk count
    (snap.cc:547-548)."""
    for name in ("test.in", "mms.in"):
        d = D.parse_deck(DECKS / name).deck
        assert d.chunks == (2, 2, 2)
        d = dataclasses.replace(d, iitm=2, oitm=2, nsteps=1) if name == "test.in" else d
        prob = P.make_problem(d)
        fc, rc = RefSnap(d).solve(prob, nthreads=4)
        f1, r1 = RefSnap(dataclasses.replace(d, chunks=(1, 1, 1))).solve(prob, nthreads=4)
        assert np.max(np.abs(fc - f1) / np.abs(f1)) < 1e-13
        assert rc["inners_per_outer"] == r1["inners_per_outer"]
        if name == "mms.in":
            assert np.isclose(rc["mms"]["sum"], r1["mms"]["sum"], rtol=1e-12)
            assert np.isclose(rc["mms"]["avg"] * 8, r1["mms"]["avg"], rtol=1e-12)
