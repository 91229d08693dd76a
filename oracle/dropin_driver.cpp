/*
 * Drop-in check (test infrastructure): the reference's own SimulationHost and scenes,
 * stepped with the CUDA backend installed as Solver::physicsBackend, against
 *   - the reference's CPU backend (list-order sweep; the reference's own GPU-vs-CPU
 *     compare gate applies: max position error < 0.05 over 120 frames), and
 *   - the reference's CPU solver run in the GPU's colour order (prepareStep, body list
 *     relinked into the sweep order read from the device, iteratePrimalDualCpu,
 *     finishStep): must be bit-identical.
 * With --commands, every host gets the same scripted bridge commands between frames
 * (drag begin / move / end, iterations, broadphase, time step, gravity); --round runs the
 * reference's scenes with spheres, capsules and cylinders (and the cloth and soft body).
 * Built by oracle/Makefile (target `dropin`) from the reference's sources plus the
 * adapter avbd_demo3d_b200/host/cuda_avbd_backend.cpp; prints one JSON line per scene.
 */
#include "cuda_avbd_backend.h"
#include "avbd_cuda.h"
#include "simulation_host.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static std::vector<Rigid *> list_of(Solver &s)
{
    std::vector<Rigid *> v;
    for (Rigid *b = s.bodies; b; b = b->next)
        v.push_back(b);
    return v;
}

static void iterate_in_order(Solver &s, const std::vector<int> &order)
{
    std::vector<Rigid *> list = list_of(s);
    std::vector<char> listed(list.size(), 0);
    std::vector<Rigid *> seq;
    for (int i : order)
    {
        seq.push_back(list[i]);
        listed[i] = 1;
    }
    for (size_t i = 0; i < list.size(); ++i)
        if (!listed[i])
            seq.push_back(list[i]);
    for (size_t i = 0; i < seq.size(); ++i)
        seq[i]->next = i + 1 < seq.size() ? seq[i + 1] : 0;
    s.bodies = seq.empty() ? 0 : seq[0];
    s.iteratePrimalDualCpu();
    for (size_t i = 0; i < list.size(); ++i)
        list[i]->next = i + 1 < list.size() ? list[i + 1] : 0;
    s.bodies = list.empty() ? 0 : list[0];
}

static bool same_bits(const void *a, const void *b, size_t n) { return std::memcmp(a, b, n) == 0; }

// The n-th dynamic body of the dense SimWorld (a drag target), or -1.
static int dynamic_body(const SimulationHost &h, int nth)
{
    const SimWorld &w = h.world();
    for (size_t id = 0; id < w.bodies.size(); ++id)
    {
        const SimBodyData &d = w.bodies[id];
        if (d.active && d.source && d.source->mass > 0.0f && nth-- == 0)
            return (int)id;
    }
    return -1;
}

// A scripted session of the bridge's commands (SimulationHost::applyCommand,
// simulation_host.cpp:121-226), given before frame f: drag one body along a path,
// release it, drag another (a new joint, possibly at the freed address), import a closed
// cube mesh as a soft lattice (simulation_host.cpp:376-493), change the iteration count,
// broadphase, time step and gravity. Returns true when the import created bodies.
static bool apply_commands(SimulationHost &h, int f, float3 &anchor)
{
    bool imported = false;
    auto cmd = [&](const char *name) {
        SimulationCommand c;
        c.command = name;
        return c;
    };
    if (f == 50)
    {
        SimulationCommand c = cmd("importMesh");
        c.meshName = "cube";
        c.meshMode = "soft";
        const float v[24] = {-1, -1, -1, 1, -1, -1, 1, 1, -1, -1, 1, -1, -1, -1, 1, 1, -1, 1, 1, 1, 1, -1, 1, 1};
        const uint32_t t[36] = {0, 2, 1, 0, 3, 2, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4,
                                1, 2, 6, 1, 6, 5, 2, 3, 7, 2, 7, 6, 3, 0, 4, 3, 4, 7};
        c.meshVertices.assign(v, v + 24);
        c.meshTriangles.assign(t, t + 36);
        c.meshPosition = float3{0.0f, 0.0f, 7.0f};
        c.hasMeshPosition = true;
        imported = h.applyCommand(c);
        h.takeOutboundMessages();
    }
    if (f == 5 || f == 70)
    {
        int id = dynamic_body(h, f == 5 ? 0 : 1);
        if (id < 0)
            return imported;
        SimulationCommand c = cmd("beginDrag");
        c.bodyId = (uint32_t)id;
        c.hasBodyId = true;
        anchor = h.world().bodies[id].source->positionLin;
        c.worldHit = anchor;
        c.hasWorldHit = true;
        c.localHit = float3{0.1f, -0.05f, 0.2f};
        c.hasLocalHit = true;
        h.applyCommand(c);
    }
    if ((f > 5 && f < 60) || (f > 70 && f < 100))
    {
        SimulationCommand c = cmd("updateDrag");
        float t = (float)(f % 60);
        c.worldTarget = float3{anchor.x + 0.03f * t, anchor.y + 0.02f * t, anchor.z + 0.04f * t};
        c.hasWorldTarget = true;
        h.applyCommand(c);
    }
    if (f == 60 || f == 100)
        h.applyCommand(cmd("endDrag"));
    if (f == 30)
    {
        SimulationCommand c = cmd("setIterations");
        c.numberValue = 7;
        c.hasNumber = true;
        h.applyCommand(c);
    }
    if (f == 45)
    {
        SimulationCommand c = cmd("setBroadphase");
        c.stringValue = "sap";
        h.applyCommand(c);
    }
    if (f == 80)
    {
        SimulationCommand c = cmd("setDt");
        c.numberValue = 1.0 / 120.0;
        c.hasNumber = true;
        h.applyCommand(c);
    }
    if (f == 90)
    {
        SimulationCommand c = cmd("setGravity");
        c.numberValue = -4.0;
        c.hasNumber = true;
        h.applyCommand(c);
    }
    return imported;
}

static double qdist(quat a, quat b)
{
    double d = 0, f = 0;
    for (int k = 0; k < 4; ++k)
    {
        d += ((double)a[k] - b[k]) * ((double)a[k] - b[k]);
        f += ((double)a[k] + b[k]) * ((double)a[k] + b[k]);
    }
    return std::sqrt(d < f ? d : f);
}

int main(int argc, char **argv)
{
    int frames = 120;
    bool commands = false;
    std::vector<std::string> names;
    for (int i = 1; i < argc; ++i)
    {
        if (!std::strcmp(argv[i], "--frames") && i + 1 < argc)
            frames = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--commands"))
            commands = true;
        else if (!std::strcmp(argv[i], "--round"))
            names = {"Sphere Stack", "Sphere Ramp", "Capsule Stack", "Capsule Ramp", "Cylinder Stack",
                     "Cylinder Ramp", "Sphere Pour on Cylinders", "Sphere Pour 5000 on Cylinders",
                     "Sphere Sphere Contact Probe", "Sphere Cylinder Contact Probe", "Sphere Capsule Contact Probe",
                     "Sphere Box Contact Probe", "Sphere Rotated Cylinder Contact Probe",
                     "Sphere Rotated Capsule Contact Probe", "Sphere Rotated Box Contact Probe",
                     "Sphere Dynamic Rotated Cylinder Contact Probe", "Sphere Dynamic Rotated Capsule Contact Probe",
                     "Sphere Dynamic Rotated Box Contact Probe", "Capsule Capsule Contact Probe",
                     "Cylinder Cylinder Contact Probe", "Capsule Cylinder Contact Probe",
                     "Rotated Capsule Cylinder Contact Probe", "Mixed Primitive Contact Probe",
                     "Capsule Box Contact Probe", "Cylinder Box Contact Probe", "Cloth", "Soft Body",
                     "Soft Body 8x8x8", "Newton's Cradle", "Mesh Torus Soft+Rigid", "Empty"};
        else
            names.push_back(argv[i]);
    }
    if (names.empty())
        names = {"Ground", "Dynamic Friction", "Static Friction", "Pyramid", "Rope", "Heavy Rope", "Spring",
                 "Spring Ratio", "Stack", "Stack Ratio", "Box Box Contact Probe", "Rotated Box Box Contact Probe",
                 "Box Cluster Contact Probe", "Bridge", "Breakable"};
    int failures = 0;
    for (const std::string &name : names)
    {
        SimulationHost gpu, cpu, colour;
        if (!gpu.loadSceneByName(name.c_str()) || !cpu.loadSceneByName(name.c_str()) ||
            !colour.loadSceneByName(name.c_str()))
        {
            std::printf("{\"scene\": \"%s\", \"error\": \"unknown scene\"}\n", name.c_str());
            failures++;
            continue;
        }
        gpu.solver().physicsBackend = makeCudaAvbdPhysicsBackend(0);
        AvbdContext *ctx = cudaAvbdBackendContext(gpu.solver().physicsBackend.get());
        int firstMismatch = -1;
        double maxPos = 0, maxRot = 0, sumSq = 0;
        long count = 0;
        float3 anchors[3] = {};
        bool imported = false;
        for (int f = 1; f <= frames; ++f)
        {
            if (commands)
            {
                imported |= apply_commands(gpu, f, anchors[0]);
                apply_commands(cpu, f, anchors[1]);
                apply_commands(colour, f, anchors[2]);
            }
            gpu.stepFrame();
            cpu.stepFrame();
            int32_t nSolve = 0;
            avbd_read_solve_order(ctx, nullptr, &nSolve);
            std::vector<int> order((size_t)nSolve);
            avbd_read_solve_order(ctx, order.data(), &nSolve);
            Solver &cs = colour.solver();
            cs.prepareStep();
            iterate_in_order(cs, order);
            cs.finishStep();
            std::vector<Rigid *> g = list_of(gpu.solver()), c = list_of(cpu.solver()), k = list_of(cs);
            for (size_t i = 0; i < g.size() && i < k.size(); ++i)
            {
                bool same = same_bits(&g[i]->positionLin, &k[i]->positionLin, 12) &&
                            same_bits(&g[i]->positionAng, &k[i]->positionAng, 16) &&
                            same_bits(&g[i]->velocityLin, &k[i]->velocityLin, 12) &&
                            same_bits(&g[i]->velocityAng, &k[i]->velocityAng, 12);
                if (!same && firstMismatch < 0)
                    firstMismatch = f;
            }
            if (g.size() != k.size() && firstMismatch < 0)
                firstMismatch = f;
            for (size_t i = 0; i < g.size() && i < c.size(); ++i)
            {
                double dx = (double)g[i]->positionLin.x - c[i]->positionLin.x;
                double dy = (double)g[i]->positionLin.y - c[i]->positionLin.y;
                double dz = (double)g[i]->positionLin.z - c[i]->positionLin.z;
                double d = std::sqrt(dx * dx + dy * dy + dz * dz);
                maxPos = d > maxPos ? d : maxPos;
                double r = qdist(g[i]->positionAng, c[i]->positionAng);
                maxRot = r > maxRot ? r : maxRot;
                sumSq += d * d;
                count++;
            }
        }
        int gm = 0, cm = 0;
        for (Force *f = gpu.solver().forces; f; f = f->next)
            gm += f->type == SIM_CONSTRAINT_MANIFOLD;
        for (Force *f = colour.solver().forces; f; f = f->next)
            cm += f->type == SIM_CONSTRAINT_MANIFOLD;
        bool exact = firstMismatch < 0 && gm == cm;
        failures += exact ? 0 : 1;
        std::printf("{\"scene\": \"%s\", \"commands\": %s, \"backend\": \"%s\", \"frames\": %d, \"bodies\": %d, \"manifolds\": %d, "
                    "\"bit_exact_vs_colour_order_reference\": %s, \"first_mismatch_frame\": %d, "
                    "\"max_position_error_vs_cpu_backend\": %.6g, \"rms_position_error_vs_cpu_backend\": %.6g, "
                    "\"max_rotation_error_vs_cpu_backend\": %.6g, \"world_uploads\": %d, \"joint_edits\": %d, "
                    "\"mesh_imported\": %s}\n",
                    name.c_str(), commands ? "true" : "false", gpu.solver().physicsBackend->name(), frames, (int)list_of(gpu.solver()).size(),
                    gm, exact ? "true" : "false", firstMismatch, maxPos, count ? std::sqrt(sumSq / count) : 0.0,
                    maxRot, cudaAvbdBackendUploads(gpu.solver().physicsBackend.get()),
                    cudaAvbdBackendJointEdits(gpu.solver().physicsBackend.get()), imported ? "true" : "false");
        std::fflush(stdout);
    }
    return failures ? 1 : 0;
}
