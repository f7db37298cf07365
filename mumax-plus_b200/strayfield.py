"""StrayField (mirror of mumaxplus/strayfield.py).

The demag field of a magnet on its own grid (Magnet.demag_field,
mumaxplus/magnet.py:555-566) is the FFT convolution of libmpx.so.  Stray fields
onto other grids are not implemented yet.
"""
from . import _abi
from .fieldquantity import FieldQuantity


class StrayField(FieldQuantity):
    """Stray field of `magnet` evaluated on `grid` (the magnet's own grid)."""

    def __init__(self, magnet, grid):
        if grid != magnet.grid:
            raise NotImplementedError("stray fields on a grid other than the source magnet's are not implemented yet")
        super().__init__(magnet, _abi.Q_DEMAG_FIELD, "demag_field", "T", 3)
        self._method = "fft"

    def set_method(self, method):
        """'fft' (default).  The direct-sum 'brute' method is not implemented."""
        if method not in ("fft", "brute"):
            raise ValueError(f"unknown stray field method '{method}'")
        if method == "brute":
            raise NotImplementedError("the brute-force stray field method is not implemented")
        self._method = method
