"""Parities of the Newell tensor that the CUDA kernel construction relies on,
checked on the FP64 oracle's Newell function (no GPU).

The pair-grid stray-field table is evaluated over absolute displacements and
expanded by parity (newell.cuh `k_newell_expand_abs`), and the self-demag kernel
spectrum is stored symmetry-reduced with sign flips of the xy, xz, yz entries
(kernels.cuh `kernel_at`).  Both assume: xx, yy, zz even in every axis; xy odd
in x and y, even in z; xz odd in x and z, even in y; yz odd in y and z, even in
x.  A component odd in an axis vanishes at zero displacement along it.  The
oracle's direct evaluations at mirrored points agree to FP64 rounding of the
integrals (about 6e-15 absolute); the expansion makes them exactly symmetric."""
import itertools

import pytest

import oracle as O

# sign of component c under the reflection of axis a (0 x, 1 y, 2 z)
ODD = {0: (), 1: (), 2: (), 3: (0, 1), 4: (0, 2), 5: (1, 2)}


@pytest.mark.parametrize("cs", [(1e-9, 1e-9, 1e-9), (2e-9, 3e-9, 1.5e-9)])
def test_newell_components_have_the_expansion_parities(cs):
    pts = [(3, 2, 1), (1, 0, 2), (5, 4, 0), (0, 3, 2), (7, 1, 3)]
    for c in range(6):
        for x, y, z in pts:
            v = O.newell(c, x, y, z, cs)
            for flips in itertools.product((1, -1), repeat=3):
                sign = 1
                for a in range(3):
                    if flips[a] < 0 and a in ODD[c]:
                        sign = -sign
                w = O.newell(c, flips[0] * x, flips[1] * y, flips[2] * z, cs)
                # the FP64 integrals cancel to ~1e-14 absolute (entries up to ~1e-2)
                assert abs(w - sign * v) < 1e-13
            for a in ODD[c]:
                if (x, y, z)[a] == 0:
                    assert abs(v) < 1e-13
