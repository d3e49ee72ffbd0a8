"""The split walk's straight moves are the face loop's own outcome (CPU,
oracle).  The FP64 replay of the split walk walks a step from a free-flight
voxel as one straight line -- reflected at mirror walls, with the origin image
mirrored, when the voxel lies at the lattice's faces -- and every other step
through the face loop.  With free flight switched off every step takes the
face loop: the two replays must agree walker by walker (voxel and face-event
sequences) and in every sum to rounding (FP64 on both sides).  Lattices with
mirror walls (where border voxels fly) and periodic walls (where only inner
voxels do), impermeable and permeable membranes, narrow pulses and PGSE."""
import numpy as np
import pytest

import pyoracle
from rms_b200 import geometry


def job(lab, *, boundary, kappa, no_flight, grad=None, npar=256, seed=7):
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, [0.0, 2.0, 1.5], [80.0, 70.0, 50.0], 1000, 2000,
                                                   kappa=kappa)
    kw = dict(grad=grad) if grad is not None else dict(bval=[1.0, 2.0], bvec=[[1, 0, 0], [0, 0.6, 0.8]])
    return pyoracle.Job(lab, dt=2e-4, tn=2000, npar=npar, res=0.1, step=step, t2_steps=t2s, pij=pij, seed=seed,
                        td=td, boundary=boundary, no_flight=no_flight, **kw)


@pytest.mark.parametrize("boundary", [pyoracle.BOUNDARY_MIRROR, pyoracle.BOUNDARY_PERIODIC])
@pytest.mark.parametrize("kappa", [0.0, 0.05])
def test_straight_moves_equal_the_face_loop(boundary, kappa):
    lab = geometry.axon_lattice(12, 14, 20, 0.1, seed=2, exterior=2, r0=0.4)
    a = pyoracle.run_oracle(job(lab, boundary=boundary, kappa=kappa, no_flight=False), trace_walkers=256, split=True)
    b = pyoracle.run_oracle(job(lab, boundary=boundary, kappa=kappa, no_flight=True), trace_walkers=256, split=True)
    assert np.array_equal(a["trace"]["voxel"], b["trace"]["voxel"])
    # a straight move records no face events; compare the positions instead
    assert np.abs(a["trace"]["pos"] - b["trace"]["pos"]).max() < 1e-9
    assert np.array_equal(a["npar_count"], b["npar_count"])
    for k in ("sig0", "dx2", "dx4", "sigre"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-10, atol=1e-12 * np.abs(b[k]).max())


def test_straight_moves_equal_the_face_loop_pgse():
    lab = geometry.axon_lattice(12, 14, 20, 0.1, seed=4, exterior=2, r0=0.45)
    g = np.array([[0.15, 0.05, 3.0, 1, 0, 0], [0.2, 0.08, 2.0, 0, 0.6, 0.8]])
    a = pyoracle.run_oracle(job(lab, boundary=0, kappa=0.02, no_flight=False, grad=g, npar=2048), nthreads=8,
                            split=True)
    b = pyoracle.run_oracle(job(lab, boundary=0, kappa=0.02, no_flight=True, grad=g, npar=2048), nthreads=8,
                            split=True)
    np.testing.assert_allclose(a["sig"], b["sig"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(a["dx4"], b["dx4"], rtol=1e-10, atol=1e-12 * np.abs(b["dx4"]).max())
