"""ksim_b200 — B200-native (sm_100a) sampling hot path of ksim.

FlatProgram -> samples, bit-exact with the reference's kokkos_sim kernel:

* :class:`B200ProgramSampler` (alias ``KokkosProgramSampler``) — drop-in for
  ``ksim.KokkosProgramSampler`` (``sample/sampler.py:46-67``);
* :mod:`ksim_b200.kokkos_sim` — drop-in for the native module ``kokkos_sim``
  (``Component(graphs, num_f)``, ``.sample``, ``.eval_abs``, ``.n_out``);
* :mod:`ksim_b200.batch` — many programs in one persistent, graph-captured launch;
* :mod:`ksim_b200.serve` — continuous-batching sample server;
* :mod:`ksim_b200.synth` — seeded synthetic FlatPrograms and known answers.

The kernels live in ``lib/libksim_b200.so`` behind the C ABI of
``include/ksim_b200.h``; there is no CPU fallback.
"""
from .program import FlatComponent, FlatProgram, FlatScalarGraph, graph_to_dict  # noqa: F401
from ._abi import RNG_PHILOX, RNG_XORSHIFT  # noqa: F401


def __getattr__(name):
    # native-backed classes load libksim_b200.so on first use
    if name in ("B200ProgramSampler", "KokkosProgramSampler"):
        from . import sampler
        return getattr(sampler, name)
    if name == "Component":
        from .kokkos_sim import Component
        return Component
    raise AttributeError(name)
