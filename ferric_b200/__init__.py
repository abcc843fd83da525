"""ferric_b200 -- B200-native density-fitting contraction core of ferric.

The DF-J/DF-K Fock build and the closed-shell RI-MP2 energy with its
3-index adjoint run in ``libferric_cuda.so`` (hand-written sm_100a kernels
behind the C ABI in ``include/ferric_cuda.h``).  This package is the host
mirror of ferric's entry points for that path:

* :mod:`ferric_b200.rimp2`     -- spin components, ``try_spin_components_on_device``,
  energy + Gamma + dE/deps;
* :mod:`ferric_b200.dfjk`      -- ``DfJ`` / ``DfK`` builders (``JBuilder`` / ``KBuilder``);
* :mod:`ferric_b200.torch_ops` -- ``RiMp2Energy`` autograd function.

Importing the package loads the library; a missing library is an ImportError.
"""
from ._lib import FcError, FcStats, init, last_error  # noqa: F401

__version__ = "0.1.0"
