"""ferric_b200 -- B200-native density-fitting contraction core of ferric.

The DF-J/DF-K Fock build and the closed-shell RI-MP2 energy with its
3-index adjoint run in ``libferric_cuda.so`` (hand-written sm_100a kernels
behind the C ABI in ``include/ferric_cuda.h``).  This package is the host
mirror of ferric's entry points for that path:

* :mod:`ferric_b200.rimp2`     -- spin components, ``try_spin_components_on_device``,
  energy + Gamma + dE/deps;
* :mod:`ferric_b200.dfjk`      -- ``DfJ`` / ``DfK`` builders (``JBuilder`` / ``KBuilder``);
* :mod:`ferric_b200.torch_ops` -- ``RiMp2Energy`` autograd function.

Importing any of those modules loads the library; a missing library is an
ImportError.  The package itself imports nothing, so ``ferric_b200.build`` can
(re)build the library in a process that has not loaded it.
"""
__version__ = "0.1.0"


def __getattr__(name):
    if name in ("FcError", "FcStats", "init", "last_error"):
        from . import _lib
        return getattr(_lib, name)
    raise AttributeError(name)
