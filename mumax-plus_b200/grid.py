"""Grid (mirror of mumaxplus/grid.py and core/grid.hpp:7-89)."""
import numbers


class Grid:
    """A box of cells: `size` (nx, ny, nz) at integer `origin`."""

    def __init__(self, size, origin=(0, 0, 0)):
        if len(size) != 3:
            raise ValueError("'size' should have three dimensions.")
        if len(origin) != 3:
            raise ValueError("'origin' should have three dimensions.")
        # the reference converts to int3 (non-integers are a TypeError) and
        # rejects negative sizes (core/grid.cu:11-17); 0 marks a non-periodic
        # mastergrid axis
        if not all(isinstance(v, numbers.Integral) for v in (*size, *origin)):
            raise TypeError("grid size and origin must be integers")
        if any(s < 0 for s in size):
            raise ValueError("The grid size should be larger than or equal to 0")
        self._size = tuple(int(s) for s in size)
        self._origin = tuple(int(o) for o in origin)

    def __repr__(self):
        return f"Grid(size={self.size}, origin={self.origin})"

    def __eq__(self, other):
        return isinstance(other, Grid) and self._size == other._size and self._origin == other._origin

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash((self._size, self._origin))

    @property
    def size(self):
        """Number of cells in the x, y and z direction."""
        return self._size

    @property
    def origin(self):
        """Origin of the grid (cells)."""
        return self._origin

    @property
    def shape(self):
        """(nz, ny, nx): the numpy shape of one component."""
        nx, ny, nz = self._size
        return (nz, ny, nx)

    @property
    def ncells(self):
        nx, ny, nz = self._size
        return nx * ny * nz

    def overlaps(self, other):
        """core/grid.hpp:91-106"""
        for a in range(3):
            lo = max(self._origin[a], other._origin[a])
            hi = min(self._origin[a] + self._size[a], other._origin[a] + other._size[a])
            if hi - lo <= 0:
                return False
        return True
