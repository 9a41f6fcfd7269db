"""snap_b200: B200-native steady-state solve path of Legion-SNAP.

The compute path is the in-tree CUDA library ``libsnap_b200.so`` behind the C
ABI of ``include/snap_b200.h``; this package is its host-side mirror of the
reference's task interface (``solver.Snap``) plus the benchmark-deck input
generator (``problem``).
"""
from . import abi, problem  # noqa: F401
from .problem import DECKS, Deck, deck, make_problem, quadrature  # noqa: F401


def __getattr__(name):
    # the solver needs torch; import it lazily so host-only users do not pay for it
    if name in ("Snap", "solver"):
        from . import solver
        return solver if name == "solver" else solver.Snap
    raise AttributeError(name)
