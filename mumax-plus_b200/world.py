"""World (mirror of mumaxplus/world.py; core/world.cpp, physics/mumaxworld.cpp).

A World owns one engine (one CUDA stream on one GPU) and one solve group: all
its magnets share the time and time step of the world's TimeSolver.
"""
import warnings

from ._engine import Engine
from .grid import Grid
from .timesolver import TimeSolver


class World:
    """A world with a given cell size, optional periodic box (mastergrid) and
    demag image repetitions (pbc_repetitions)."""

    _DFT_MODES = {"fp32": 0, "tf32x3": 1}

    def __init__(self, cellsize, pbc_repetitions=(0, 0, 0), mastergrid=Grid((0, 0, 0)), device=None,
                 demag_dft="fp32"):
        """demag_dft (no counterpart in the reference, which calls cuFFT): the
        arithmetic of the y transforms of the demag convolution, "fp32"
        (shared-memory FFTs on the CUDA cores, the default) or "tf32x3"
        (tensor-core DFT GEMMs with 3xTF32 split products for y lengths 1024
        and 2048 of the padded grid)."""
        if demag_dft not in self._DFT_MODES:
            raise ValueError(f"demag_dft must be one of {sorted(self._DFT_MODES)}")
        if len(cellsize) != 3:
            raise ValueError("'cellsize' should have three dimensions.")
        if len(pbc_repetitions) != 3:
            raise ValueError("'pbc_repetitions' should have three dimensions.")
        if not all(isinstance(item, int) for item in pbc_repetitions):
            raise ValueError("All elements of `pbc_repetitions` must be integers.")
        if any(c <= 0 for c in cellsize):
            raise ValueError("The cell size should be larger than 0")
        self._cellsize = tuple(float(c) for c in cellsize)
        self._check_pbc(mastergrid, pbc_repetitions)
        self._pbc = tuple(int(p) for p in pbc_repetitions)
        self._mastergrid = Grid(mastergrid.size, mastergrid.origin)
        self._engine = Engine(device)
        self._engine.set_dft(self._DFT_MODES[demag_dft])
        self._demag_dft = demag_dft
        self._group = self._engine.group_create()
        self._relax_threshold = -1.0
        self._magnets = {}
        self._bias = (0.0, 0.0, 0.0)
        self._unnamed = 1
        self._timesolver = TimeSolver(self)

    def __repr__(self):
        return f"World(cellsize={self.cellsize})"

    @property
    def demag_dft(self):
        """Arithmetic of the demag y transforms ("fp32" or "tf32x3"), fixed at construction."""
        return self._demag_dft

    # ------------------------------------------------------------- internals
    @staticmethod
    def _check_pbc(mastergrid, pbc):
        """core/world.cpp checkPbcRepetitions / checkPbcCompatibility"""
        if any(p < 0 for p in pbc):
            raise ValueError("Number of pbcRepetitions should not be negative.")
        for a in range(3):
            if (mastergrid.size[a] == 0) != (pbc[a] == 0):
                raise ValueError("0 in size of mastergrid should match 0 in pbcRepetitions.")

    def _in_mastergrid(self, grid):
        mg = self._mastergrid
        for a in range(3):
            if mg.size[a] > 0:
                d1 = grid.origin[a] - mg.origin[a]
                d2 = d1 + grid.size[a] - mg.size[a]
                if d1 < 0 or d2 > 0:
                    return False
        return True

    def _check_addibility(self, grid, name):
        """physics/mumaxworld.cpp:35-55"""
        if not self._in_mastergrid(grid):
            raise IndexError("Can not add magnet because the grid does not fit in the mastergrid ")
        for m in self._magnets.values():
            if grid.overlaps(m.grid):
                raise IndexError("Can not add magnet because it overlaps with another magnet.")
        if name and name in self._magnets:
            raise RuntimeError(f"A magnet with the name '{name}' already exists")

    def _next_name(self):
        name = f"ferromagnet_{self._unnamed}"
        self._unnamed += 1
        return name

    def _register(self, magnet):
        self._magnets[magnet.name] = magnet

    def _update_all(self):
        for m in self._magnets.values():
            m._update()

    # ------------------------------------------------------------- API
    @property
    def timesolver(self):
        return self._timesolver

    @property
    def cellsize(self):
        return self._cellsize

    @property
    def bias_magnetic_field(self):
        return self._bias

    @bias_magnetic_field.setter
    def bias_magnetic_field(self, value):
        v = tuple(float(x) for x in value)
        if len(v) != 3:
            raise ValueError("the bias field needs three components")
        self._bias = v
        self._engine.set_world_bias(v)

    @property
    def ferromagnets(self):
        return dict(self._magnets)

    def get_ferromagnet(self, name):
        if name not in self._magnets:
            raise KeyError(f"No magnet named {name}")
        return self._magnets[name]

    @property
    def mastergrid(self):
        return self._mastergrid

    @mastergrid.setter
    def mastergrid(self, mastergrid):
        self._check_pbc(mastergrid, self._pbc)
        self._mastergrid = Grid(mastergrid.size, mastergrid.origin)
        self._check_all_in_mastergrid()
        self._update_all()

    @property
    def pbc_repetitions(self):
        return self._pbc

    @pbc_repetitions.setter
    def pbc_repetitions(self, value):
        if len(value) != 3:
            raise ValueError("'pbc_repetitions' should have three dimensions.")
        if not all(isinstance(item, int) for item in value):
            raise ValueError("All elements of `pbc_repetitions` must be integers.")
        self._check_pbc(self._mastergrid, value)
        self._pbc = tuple(value)
        self._update_all()

    def _check_all_in_mastergrid(self):
        for m in self._magnets.values():
            if not self._in_mastergrid(m.grid):
                raise IndexError("Not all magnets of the world fit inside the mastergrid.")

    @property
    def bounding_grid(self):
        """Smallest grid containing all magnets (physics/mumaxworld.cpp boundingGrid)."""
        if not self._magnets:
            raise IndexError("Cannot find minimum bounding box if there are no magnets in the world.")
        grids = [m.grid for m in self._magnets.values()]
        lo = [min(g.origin[a] for g in grids) for a in range(3)]
        hi = [max(g.origin[a] + g.size[a] for g in grids) for a in range(3)]
        return Grid([hi[a] - lo[a] for a in range(3)], lo)

    def set_pbc(self, pbc_repetitions, mastergrid=None):
        """Set the periodic boundary conditions (physics/mumaxworld.cpp setPBC)."""
        if len(pbc_repetitions) != 3:
            raise ValueError("'pbc_repetitions' should have three dimensions.")
        if not all(isinstance(item, int) for item in pbc_repetitions):
            raise ValueError("All elements of `pbc_repetitions` must be integers.")
        if any(p < 0 for p in pbc_repetitions):
            raise ValueError("Number of pbcRepetitions should not be negative.")
        if mastergrid is None:
            bg = self.bounding_grid
            size = [bg.size[a] if pbc_repetitions[a] != 0 else 0 for a in range(3)]
            mastergrid = Grid(size, bg.origin)
        self._check_pbc(mastergrid, pbc_repetitions)
        self._pbc = tuple(int(p) for p in pbc_repetitions)
        self._mastergrid = Grid(mastergrid.size, mastergrid.origin)
        self._check_all_in_mastergrid()
        self._update_all()

    def unset_pbc(self):
        self._pbc = (0, 0, 0)
        self._mastergrid = Grid((0, 0, 0))
        self._update_all()

    def relax(self, tol=1e-9):
        """Relax all magnets of the world to an energy minimum
        (mumaxplus/world.py:117-141, physics/relaxer.cpp)."""
        if tol >= 1e-5:
            warnings.warn("The set tolerance is greater than or equal to the default value"
                           + " used for the timesolver (1e-5). Using this value results"
                           + " in no torque minimization, only energy minimization.", UserWarning)
        self._engine.relax(self._group, tol, self._relax_threshold)

    def minimize(self, tol=1e-6, nsamples=10):
        """Minimize the total energy of the world (mumaxplus/world.py:95-115)."""
        self._engine.minimize(self._group, tol, nsamples)

    def save_state(self):
        """Checkpoint of the time integration (no counterpart in mumax+): time,
        time step, step count and, for every magnet, m and the Dormand-Prince
        FSAL derivative, as a uint8 array.  load_state() into a world with
        magnets of the same sizes continues exactly as this one would."""
        return self._engine.group_save(self._group)

    def load_state(self, state):
        self._engine.group_load(self._group, state)

    @property
    def RelaxTorqueThreshold(self):
        """Threshold torque for relax (default -1, see Ferromagnet.RelaxTorqueThreshold)."""
        return self._relax_threshold

    @RelaxTorqueThreshold.setter
    def RelaxTorqueThreshold(self, value):
        assert value != 0, "The relax threshold should not be zero."
        self._relax_threshold = float(value)
