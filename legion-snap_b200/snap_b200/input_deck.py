"""The reference's input decks (input/*.in) and its convergence/timing log.

``parse_deck`` reads a deck as Snap::parse_arguments does (snap.cc:1032-1168):
two header lines, then ``name=value`` entries in a fixed order, with the same
validity checks (raised as ``ValueError`` instead of the reference's
``assert``/``exit``).  ``run_deck`` solves it through the C ABI and prints the
reference's log: the argument report (snap.cc:1345-1380), one line per inner
and outer iteration and per time step, and the execution summary
(convergence.cc:154-264, times measured on the host around each iteration).

The chunk counts (npey, npez, ichunk) describe the reference's spatial
decomposition into Legion tasks; this build sweeps the whole mesh as one
domain on one GPU, which gives the same solution, so they are read, checked
and reported but do not change the computation.
"""
from __future__ import annotations

import dataclasses
import pathlib
import re
import sys

from .problem import Deck

# (name, kind) in the order parse_arguments reads them (snap.cc:1042-1109)
FIELDS = [
    ("npey", int), ("npez", int), ("ichunk", int), ("nthreads", int), ("nnested", int),
    ("ndimen", int), ("nx", int), ("lx", float), ("ny", int), ("ly", float), ("nz", int),
    ("lz", float), ("nmom", int), ("nang", int), ("ng", int), ("epsi", float), ("iitm", int),
    ("oitm", int), ("timedep", int), ("tf", float), ("nsteps", int), ("mat_opt", int),
    ("src_opt", int), ("scatp", int), ("it_det", int), ("fluxp", int), ("fixup", int),
    ("soloutp", int), ("kplane", int), ("popout", int), ("swp_typ", int), ("angcpy", int),
]

MATERIAL_LAYOUTS = {0: "Homogenous Layout", 1: "Center Layout", 2: "Corner Layout"}
SOURCE_LAYOUTS = {0: "Everywhere", 1: "Center", 2: "Corner", 3: "MMS"}


@dataclasses.dataclass
class DeckFile:
    """Every entry of a deck, and the solver's view of it (``deck``)."""
    values: dict
    deck: Deck
    path: str = ""


def _entries(text: str):
    lines = text.splitlines()
    if len(lines) < 2:
        raise ValueError("a deck has two header lines before its entries")
    body = "\n".join(lines[2:])
    return re.findall(r"([A-Za-z_]\w*)\s*=\s*([-+0-9.eEdD]+)", body)


def parse_deck_text(text: str, path: str = "") -> DeckFile:
    entries = _entries(text)
    vals = {}
    for i, (name, kind) in enumerate(FIELDS):
        if i >= len(entries) or entries[i][0] != name:
            found = entries[i][0] if i < len(entries) else "end of deck"
            raise ValueError(f"expected '{name}=' as entry {i + 1}, found {found}")
        raw = entries[i][1].replace("d", "e").replace("D", "E")
        vals[name] = kind(float(raw)) if kind is int else float(raw)
    v = vals
    # snap.cc:1110-1160
    if v["angcpy"] == 1:
        raise ValueError("angcpy=1 is not supported (two copies of the angular flux are kept)")
    if not v["swp_typ"]:
        raise ValueError("swp_typ=0 is not supported (mini-KBA sweeps only)")
    if v["mat_opt"] not in MATERIAL_LAYOUTS:
        raise ValueError(f"mat_opt={v['mat_opt']} is not a layout")
    if v["src_opt"] not in SOURCE_LAYOUTS:
        raise ValueError(f"src_opt={v['src_opt']} is not a layout")
    checks = [
        (v["ndimen"] == 3, "ndimen must be 3 (the sweep is three-dimensional, sweep.cc:253)"),
        (1 <= v["ichunk"] <= v["nx"], "1 <= ichunk <= nx"),
        (1 <= v["npey"] <= v["ny"], "1 <= npey <= ny"),
        (1 <= v["npez"] <= v["nz"], "1 <= npez <= nz"),
        (v["nx"] >= 4 and v["ny"] >= 4 and v["nz"] >= 4, "nx, ny, nz >= 4"),
        (v["lx"] > 0 and v["ly"] > 0 and v["lz"] > 0, "lx, ly, lz > 0"),
        (v["nx"] % v["ichunk"] == 0, "nx % ichunk == 0"),
        (v["ny"] % v["npey"] == 0, "ny % npey == 0"),
        (v["nz"] % v["npez"] == 0, "nz % npez == 0"),
        (1 <= v["nmom"] <= 4, "1 <= nmom <= 4"),
        (v["nang"] >= 1 and v["ng"] >= 1, "nang, ng >= 1"),
        (0.0 < v["epsi"] < 1e-2, "0 < epsi < 1e-2"),
        (v["iitm"] >= 1 and v["oitm"] >= 1, "iitm, oitm >= 1"),
        (not v["timedep"] or v["tf"] >= 0.0, "tf >= 0 when timedep"),
        (v["nsteps"] >= 1, "nsteps >= 1"),
    ]
    for ok, msg in checks:
        if not ok:
            raise ValueError(f"invalid deck: {msg}")
    d = Deck(v["nx"], v["ny"], v["nz"], nang=v["nang"], ng=v["ng"], nmom=v["nmom"],
             epsi=v["epsi"], iitm=v["iitm"], oitm=v["oitm"], fixup=bool(v["fixup"]),
             lx=v["lx"], ly=v["ly"], lz=v["lz"], timedep=bool(v["timedep"]), tf=v["tf"],
             nsteps=v["nsteps"], mat_opt=v["mat_opt"], src_opt=v["src_opt"],
             chunks=(v["npey"], v["npez"], v["ichunk"]))
    return DeckFile(vals, d, path)


def parse_deck(path) -> DeckFile:
    p = pathlib.Path(path)
    return parse_deck_text(p.read_text(), str(p))


def report_arguments(df: DeckFile, out=None):
    """The argument report of Snap::report_arguments (snap.cc:1345-1380)."""
    out = sys.stdout if out is None else out
    v = df.values
    yn = lambda b: "Yes" if b else "No"  # noqa: E731
    lines = [
        f"Dimensions: {v['ndimen']}", f"X-Chunks: {v['ichunk']}", f"Y-Chunks: {v['npey']}",
        f"Z-Chunks: {v['npez']}", f"nx,ny,nz: {v['nx']},{v['ny']},{v['nz']}",
        f"lx,ly,lz: {v['lx']:.8g},{v['ly']:.8g},{v['lz']:.8g}", f"Moments: {v['nmom']}",
        f"Angles: {v['nang']}", f"Groups: {v['ng']}", f"Convergence: {v['epsi']:.8g}",
        f"Max Inner Iterations: {v['iitm']}", f"Max Outer Iterations: {v['oitm']}",
        f"Time Dependent: {yn(v['timedep'])}", f"Total Simulation Time: {v['tf']:.8g}",
        f"Total Steps: {v['nsteps']}", f"Material Layout: {MATERIAL_LAYOUTS[v['mat_opt']]}",
        f"Source Layout: {SOURCE_LAYOUTS[v['src_opt']]}", f"Dump Scatter: {yn(v['scatp'])}",
        f"Dump Iteration: {yn(v['it_det'])}",
        "Dump Flux: " + {2: "All", 1: "Scalar"}.get(v["fluxp"], "No"),
        f"Fixup Flux: {yn(v['fixup'])}", f"Dump Solution: {yn(v['soloutp'])}",
        f"Dump Kplane: {v['kplane']}",
        "Dump Population: " + {2: "All", 1: "Final"}.get(v["popout"], "No"),
        f"Mini-KBA Sweep: {yn(v['swp_typ'])}", f"Single Angle Copy: {yn(v['angcpy'] == 1)}",
    ]
    for line in lines:
        print(line, file=out)


def convergence_log(records, out=None):
    """The per-iteration lines and the summary of the reference's convergence
    monad (convergence.cc:154-264) from the solve's iteration records
    (dicts with kind 'inner'/'outer', time_step, outer, inner, converged, us).
    Outer iteration 0 of a time step has no outer test (snap.cc:521-522), so
    it prints no outer line, as in the reference."""
    out = sys.stdout if out is None else out
    total_inner = total_outer = 0
    inner_us = outer_us = step_us = total_step_us = 0.0
    steps = 0
    for r in records:
        if r["kind"] == "inner":
            state = "CONVERGED" if r["converged"] else "did not converge"
            print(f"Inner loop {r['inner']} of outer loop {r['outer']} of time step "
                  f"{r['time_step']} {state} in {int(r['us'])} microseconds", file=out)
            total_inner += 1
            inner_us += r["us"]
            step_us += r["us"]
        else:
            if r["converged"]:
                print(f"Outer loop {r['outer']} of time step {r['time_step']} CONVERGED in "
                      f"{int(r['us'])} microseconds", file=out)
                print(f"Time step {r['time_step']} took {int(step_us)} microseconds", file=out)
                total_step_us += step_us
                step_us = 0.0
                steps += 1
            else:
                print(f"Outer loop {r['outer']} of time step {r['time_step']} did not converge "
                      f"in {int(r['us'])} microsecond", file=out)
            total_outer += 1
            outer_us += r["us"]
    bar = "-" * 57
    print(bar, file=out)
    print("SNAP Execution Summary", file=out)
    print(bar, file=out)
    print(f"  Execution Time: {int(total_step_us)} us", file=out)
    print(f"  Total Time Steps: {steps} (avg {total_step_us / max(steps, 1):.8g} us / iter)",
          file=out)
    print(f"  Total Outer Loops: {total_outer} (avg {outer_us / max(total_outer, 1):.8g} us / "
          f"iter)", file=out)
    print(f"  Total Inner Loops: {total_inner} (avg {inner_us / max(total_inner, 1):.8g} us / "
          f"iter)", file=out)
    print(bar, file=out)


def run_deck(path, device: int = 0, out=None):
    """Solves a reference deck through the C ABI on one GPU and prints the
    reference's argument report and convergence/timing log.  Returns the
    flux moments [G, C, cmom] (a CUDA tensor) and the iteration record."""
    from .solver import Snap
    from .problem import make_problem
    out = sys.stdout if out is None else out
    df = parse_deck(path)
    d = df.deck
    if d.src_opt == 3:
        from .mms import run_mms
        return run_mms(d, device=device, out=out)
    report_arguments(df, out)
    snap = Snap(d, device=device)
    try:
        flux, rec = snap.transport_solve(snap.device_problem(make_problem(d)))
    finally:
        snap.close()
    convergence_log(rec["records"], out)
    return flux, rec


if __name__ == "__main__":
    run_deck(sys.argv[1])
