"""B200 RK4 / JST / viscous hot path of the 2-D / axisymmetric turbulent Navier-Stokes
solver: C-ABI binding (``_lib``), host-side solver mirror (``solver``), case files
(``formats``) and structured case generators (``cases``)."""
from . import cases, formats  # noqa: F401
