"""TimeSolver (mirror of mumaxplus/timesolver.py).

Stepping runs in libmpx.so: TimeSolver::step / steps / run of
core/timesolver.cpp:77-111 with the adaptive Runge-Kutta stepper of
core/rungekutta.cpp:25-151, the accept/reject decision and the new time step
taken on the GPU in FP64.
"""
import os as _os

from . import _abi


class TimeSolverOutput:
    """Values of quantities collected at time points (optionally written as TSV)."""

    def __init__(self, quantity_dict, file_name=None):
        self._quantities = quantity_dict
        self._data = {"time": []}
        for key in self._quantities.keys():
            self._data[key] = []
        self._keys = list(self._data.keys())
        self._file_name = file_name
        if self._file_name is not None:
            directory = _os.path.dirname(self._file_name)
            if directory:
                _os.makedirs(directory, exist_ok=True)
            with open(self._file_name, "w") as f:
                print("# " + "\t".join(self._keys), file=f)

    def write_line(self, time):
        self._append(time, {key: func() for key, func in self._quantities.items()})

    def _append(self, time, values):
        self._data["time"].append(time)
        for key in self._quantities.keys():
            self._data[key].append(values[key])
        if self._file_name is not None:
            with open(self._file_name, "a") as f:
                print(*[self._data[key][-1] for key in self._keys], sep="\t", file=f)

    def __getitem__(self, key):
        return self._data[key]


class TimeSolver:
    """Evolves a World in time; every World has one (world.timesolver)."""

    def __init__(self, world):
        self._world = world

    @property
    def _e(self):
        return self._world._engine

    @property
    def _g(self):
        return self._world._group

    def _params(self):
        return self._e.solver_params(self._g)

    def _set(self, **kw):
        p = self._params()
        for k, v in kw.items():
            setattr(p, k, v)
        self._e.set_solver_params(self._g, p)

    def _assure_sensible_timestep(self):
        """mumaxplus/timesolver.py:61-70"""
        if self.adaptive_timestep:
            s = self.sensible_timestep
            if self.timestep == 0.0 or self.timestep > s:
                self.timestep = s

    def set_method(self, method_name):
        """'Heun', 'BogackiShampine', 'CashKarp', 'Fehlberg' (default) or 'DormandPrince'."""
        if not isinstance(method_name, str):
            raise TypeError("the method name should be a string")
        if method_name not in _abi.RK_METHODS:
            raise ValueError(f"'{method_name}' is not a valid Runge Kutta method name")
        self._set(method=_abi.RK_METHODS[method_name])

    @property
    def method(self):
        return _abi.RK_NAMES[self._params().method]

    def step(self):
        self._e.step(self._g)

    def steps(self, nsteps):
        self._assure_sensible_timestep()
        self._e.steps(self._g, nsteps)

    def run_while(self, condition):
        self._assure_sensible_timestep()
        while condition():
            self._e.step(self._g)

    def run(self, duration):
        self._assure_sensible_timestep()
        self._e.run(self._g, duration)

    def solve(self, timepoints, quantity_dict, file_name=None, tqdm=False):
        """Run to each time point and record the quantities there."""
        timepoints = list(timepoints)
        assert all(i1 <= i2 for i1, i2 in zip(timepoints, timepoints[1:])), \
            "The list of timepoints should be increasing."
        assert self.time <= timepoints[0], "The list of timepoints should lie in the future."
        self._assure_sensible_timestep()
        output = TimeSolverOutput(quantity_dict, file_name)
        cols = self._magnetization_columns(quantity_dict)
        if cols is not None:  # sampled on the device, one table back at the end
            table = self._e.run_sampled(self._g, timepoints, len(self._world._magnets))
            for row in table:
                output._append(float(row[0]), {k: [float(v) for v in row[c:c + 3]] for k, c in cols.items()})
            return output
        it = timepoints
        if tqdm:
            from tqdm import tqdm as _tqdm
            it = _tqdm(timepoints)
        for tp in it:
            self._e.run(self._g, tp - self.time)
            output.write_line(self.time)
        return output

    def _magnetization_columns(self, quantity_dict):
        """Column of each quantity in the device-sampled table when every one is
        the average magnetization of a magnet of this world (the bound method
        `magnet.magnetization.average`), else None (other callables are
        evaluated on the host at every time point)."""
        from .fieldquantity import FieldQuantity
        from .parameter import Variable

        order = {id(m): j for j, m in enumerate(self._world._magnets.values())}
        cols = {}
        for key, func in quantity_dict.items():
            obj, fn = getattr(func, "__self__", None), getattr(func, "__func__", None)
            if isinstance(obj, Variable) and fn is Variable.average:
                magnet = obj._magnet
            elif (isinstance(obj, FieldQuantity) and fn is FieldQuantity.average
                  and obj._q == _abi.Q_MAGNETIZATION):
                magnet = obj._magnet
            else:
                return None
            j = order.get(id(magnet))
            if j is None:
                return None
            cols[key] = 1 + 3 * j
        return cols

    # -------------------------------------------------------- properties
    @property
    def sensible_timestep(self):
        return self._e.sensible_timestep(self._g)

    @property
    def timestep(self):
        return self._e.get_timestep(self._g)

    @timestep.setter
    def timestep(self, dt):
        self._e.set_timestep(self._g, dt)

    @property
    def adaptive_timestep(self):
        return bool(self._params().adaptive)

    @adaptive_timestep.setter
    def adaptive_timestep(self, adaptive):
        self._set(adaptive=1 if adaptive else 0)

    @property
    def time(self):
        return self._e.get_time(self._g)

    @time.setter
    def time(self, t):
        self._e.set_time(self._g, t)

    @property
    def max_error(self):
        return self._params().max_error

    @max_error.setter
    def max_error(self, error):
        assert error > 0, "The maximum error should be bigger than 0."
        self._set(max_error=float(error))

    @property
    def headroom(self):
        return self._params().headroom

    @headroom.setter
    def headroom(self, h):
        assert h > 0, "The headroom should be bigger than 0."
        self._set(headroom=float(h))

    @property
    def lower_bound(self):
        return self._params().lower_bound

    @lower_bound.setter
    def lower_bound(self, v):
        assert v > 0, "The lower bound should be bigger than 0."
        p = self._params()
        p.lower_bound = float(v)
        self._e.set_solver_params(self._g, p) if p.lower_bound < p.upper_bound else self._store_bounds(p)

    @property
    def upper_bound(self):
        return self._params().upper_bound

    @upper_bound.setter
    def upper_bound(self, v):
        assert v > 0, "The upper bound should be bigger than 0."
        p = self._params()
        p.upper_bound = float(v)
        self._e.set_solver_params(self._g, p) if p.lower_bound < p.upper_bound else self._store_bounds(p)

    def _store_bounds(self, p):
        # the reference accepts crossed bounds at set time and raises when adapting
        raise RuntimeError("The lower bound should be lower than the upper bound.")

    @property
    def sensible_factor(self):
        return self._params().sensible_factor

    @sensible_factor.setter
    def sensible_factor(self, f):
        assert f > 0, "The sensible factor should be bigger than 0."
        self._set(sensible_factor=float(f))

    @property
    def sensible_timestep_default(self):
        return self._params().sensible_timestep_default

    @sensible_timestep_default.setter
    def sensible_timestep_default(self, dt):
        self._set(sensible_timestep_default=float(dt))
