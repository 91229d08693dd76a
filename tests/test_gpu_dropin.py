"""The drop-in: the reference's own SimulationHost scenes stepped with the CUDA backend
installed as Solver::physicsBackend (the C++ adapter in avbd_demo3d_b200/host), checked
against the reference's CPU solver in the GPU's colour order (bit-exact) and against its
CPU backend (the reference's GPU-vs-CPU compare gate: max position error < 0.05 over
120 frames on Pyramid and Rope, viewer/package.json:24)."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "avbd_dropin")


def test_reference_scenes_through_the_backend_adapter(gpu):
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in harness not built (needs the reference sources: make -C oracle dropin)")
    out = subprocess.run([DROPIN, "--frames", "120"], capture_output=True, text=True, timeout=600)
    rows = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(rows) == 15, out.stdout + out.stderr
    for r in rows:
        assert r["backend"].startswith("CUDA AVBD"), r
        assert r["bit_exact_vs_colour_order_reference"], r
    gates = {r["scene"]: r for r in rows}
    for scene in ("Pyramid", "Rope"):
        assert gates[scene]["max_position_error_vs_cpu_backend"] < 0.05, gates[scene]
    assert out.returncode == 0, out.stderr


def test_bridge_commands_through_the_backend_adapter(gpu):
    """The bridge's commands between frames on every scene (drag begin / move / end twice,
    importMesh of a closed cube as a soft sphere lattice, setIterations, setBroadphase sap,
    setDt, setGravity): the adapter turns the drag joint's
    creation, anchor moves and deletion into device joint edits and stays bit-exact with
    the reference's CPU solver in the GPU's colour order."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in harness not built (needs the reference sources: make -C oracle dropin)")
    out = subprocess.run([DROPIN, "--frames", "120", "--commands"], capture_output=True, text=True, timeout=600)
    rows = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(rows) == 15, out.stdout + out.stderr
    for r in rows:
        assert r["commands"] and r["backend"].startswith("CUDA AVBD"), r
        assert r["bit_exact_vs_colour_order_reference"], r
        # drags are joint edits, not reloads; the mesh import adds bodies and reloads once
        assert r["world_uploads"] == 1 + (1 if r["mesh_imported"] else 0), r
    dragged = [r for r in rows if r["joint_edits"] > 0]
    assert len(dragged) >= 10, rows  # every scene with a dynamic body was dragged
    assert sum(r["mesh_imported"] for r in rows) >= 10, rows  # the cube lattice was built
    assert out.returncode == 0, out.stderr


def test_round_shape_scenes_through_the_backend_adapter(gpu):
    """The reference's scenes with spheres, capsules and cylinders (stacks, ramps, the sphere
    pours on cylinders, every contact probe, Newton's cradle, the mesh-lattice torus), the
    sphere cloth and the soft bodies: the round
    narrowphase, contact offsets and sphere rolling friction on the GPU stay bit-exact with
    the reference's CPU solver in the GPU's colour order."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in harness not built (needs the reference sources: make -C oracle dropin)")
    out = subprocess.run([DROPIN, "--frames", "120", "--round"], capture_output=True, text=True, timeout=1200)
    rows = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(rows) == 31, out.stdout + out.stderr
    for r in rows:
        assert r["backend"].startswith("CUDA AVBD"), r
        assert r["bit_exact_vs_colour_order_reference"], r
    assert out.returncode == 0, out.stderr


def test_sphere_pour_20000(gpu):
    """The largest reference scene (20,000 spheres poured on cylinders) for its first 20
    frames, bit-exact in the GPU's colour order."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in harness not built (needs the reference sources: make -C oracle dropin)")
    out = subprocess.run([DROPIN, "--frames", "20", "Sphere Pour 20000 on Cylinders"], capture_output=True, text=True,
                         timeout=1200)
    rows = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(rows) == 1 and rows[0]["bodies"] > 20000, out.stdout + out.stderr
    assert rows[0]["bit_exact_vs_colour_order_reference"], rows[0]
