"""The force plug-in: mpm_add_grid_forces hands the grid update the node forces of
a force the library does not model, as a PhysBAM scene adds any
PARTICLE_GRID_FORCES (Hybrid_Methods/Forces/PARTICLE_GRID_FORCES.h:17-36) to
MPM_EXAMPLE::forces (MPM_EXAMPLE.cpp:115-153).

The fixture small3d_node_force is the reference's own driver with such a force
(a constant vector at every node with mass, oracle/ref_scene.h
NODE_FORCE_CONSTANT) among its forces; the driver evaluates the same force and
passes it between mpm_particle_to_grid and mpm_apply_forces.  Its parity with
the reference runs with the other fixtures in test_gpu_parity.py (plain FP64
and fast FP32 in every launch shape); here, the order the entry point needs."""
import pytest

from make_golden import load

pytestmark = pytest.mark.gpu


def D():
    from physbam_b200 import driver
    return driver


def test_node_force_out_of_order_is_refused(cuda_device):
    scene, _ = load("small3d_node_force")
    drv = D().MPM_DRIVER(scene, precision=D().FP32, path=D().PATH_FAST)
    drv.set_scene_particles(scene)
    f = drv._node_force_array()
    with pytest.raises(D().MPMError) as e:      # before P2G
        drv.add_grid_forces(f)
    assert e.value.code == 7
    drv.Particle_To_Grid()
    drv.add_grid_forces(f)
    drv.Apply_Forces()
    with pytest.raises(D().MPMError) as e:      # after the grid update
        drv.add_grid_forces(f)
    assert e.value.code == 7
    with pytest.raises(ValueError):
        drv.add_grid_forces(f[:, :, :, :2])
    drv.close()
