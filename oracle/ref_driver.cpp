/*
 * Driver around the REFERENCE solver, compiled together with the reference's own
 * sources by oracle/Makefile into oracle/_ref/libavbd_ref.so (test infrastructure).
 *
 * It builds a scene through the reference's public constructors (Rigid, Joint,
 * Spring, IgnoreCollision; solver.h:221, 262, 276, 288), steps it with the stock
 * CPU backend (Solver::step -> CpuReferenceBackend, solver.cpp:664-674, 934-937)
 * or with the phased API (prepareStep / iteratePrimalDualCpu / finishStep,
 * solver.h:399-401), and reads state back in list order. The exported functions
 * mirror oracle/avbd_oracle.h with a `ref_` prefix so the tests can run both.
 *
 * Colour-order stepping relinks Solver::bodies (Rigid::next, solver.h:202, 357)
 * into a caller-given sweep order between prepareStep and iteratePrimalDualCpu and
 * restores the original list afterwards; nothing else in the reference changes.
 */
#include "solver.h"

#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace
{
struct RefWorld
{
    Solver solver;
    std::vector<Rigid *> list; // list order: index 0 = solver.bodies head
    std::unordered_map<const Rigid *, int> index;
    std::vector<Joint *> added; // joints created between steps, by handle
};

void rebuild_index(RefWorld *w)
{
    w->list.clear();
    w->index.clear();
    for (Rigid *b = w->solver.bodies; b != 0; b = b->next)
    {
        w->index[b] = (int)w->list.size();
        w->list.push_back(b);
    }
}

struct RefParams
{
    float dt;
    float gravity;
    int iterations;
    float alpha;
    float betaLin;
    float betaAng;
    float gamma;
    int broadphase;
    int orderMode;
};

void apply_params(Solver &s, const RefParams *p)
{
    s.dt = p->dt;
    s.gravity = p->gravity;
    s.iterations = p->iterations;
    s.alpha = p->alpha;
    s.betaLin = p->betaLin;
    s.betaAng = p->betaAng;
    s.gamma = p->gamma;
    s.broadphaseMode = p->broadphase == 0   ? BROADPHASE_ALL_PAIRS
                       : p->broadphase == 2 ? BROADPHASE_SWEEP_AND_PRUNE
                                            : BROADPHASE_UNIFORM_GRID;
}

template <typename T>
std::vector<T *> forces_of_type(RefWorld *w, SimConstraintType type)
{
    // solver.forces is newest first; return creation order
    std::vector<T *> out;
    for (Force *f = w->solver.forces; f != 0; f = f->next)
        if (f->type == type)
            out.push_back((T *)f);
    return std::vector<T *>(out.rbegin(), out.rend());
}
} // namespace

extern "C"
{

/* shape (creation order, NULL = all boxes): 0 box (size3), 1 sphere, 2 capsule, 3 cylinder,
 * built with the reference's Rigid::makeSphere / makeCapsule / makeCylinder from
 * dim2 = (radius, halfLength). */
void *ref_create_shapes(const RefParams *params, int nBodies, const int *shape, const float *dim2,
                        const float *size3, const float *density, const float *friction, const float *pos3,
                        const float *vel3, const float *quat4, int nForces, const int *ftype, const int *fa,
                        const int *fb, const float *frA3, const float *frB3, const float *fparam3)
{
    RefWorld *w = new RefWorld();
    apply_params(w->solver, params);
    std::vector<Rigid *> created;
    for (int c = 0; c < nBodies; ++c)
    {
        float3 pos = float3{pos3[3 * c], pos3[3 * c + 1], pos3[3 * c + 2]};
        float3 vel = float3{vel3[3 * c], vel3[3 * c + 1], vel3[3 * c + 2]};
        int t = shape ? shape[c] : 0;
        Rigid *r;
        if (t == 1)
            r = Rigid::makeSphere(&w->solver, dim2[2 * c], density[c], friction[c], pos, vel);
        else if (t == 2)
            r = Rigid::makeCapsule(&w->solver, dim2[2 * c], dim2[2 * c + 1], density[c], friction[c], pos, vel);
        else if (t == 3)
            r = Rigid::makeCylinder(&w->solver, dim2[2 * c], dim2[2 * c + 1], density[c], friction[c], pos, vel);
        else
            r = new Rigid(&w->solver, float3{size3[3 * c], size3[3 * c + 1], size3[3 * c + 2]}, density[c],
                          friction[c], pos, vel);
        r->positionAng = quat{quat4[4 * c], quat4[4 * c + 1], quat4[4 * c + 2], quat4[4 * c + 3]};
        created.push_back(r);
    }
    for (int k = 0; k < nForces; ++k)
    {
        Rigid *a = fa[k] >= 0 ? created[fa[k]] : 0;
        Rigid *b = created[fb[k]];
        float3 rA = {frA3[3 * k], frA3[3 * k + 1], frA3[3 * k + 2]};
        float3 rB = {frB3[3 * k], frB3[3 * k + 1], frB3[3 * k + 2]};
        if (ftype[k] == 1)
            new Joint(&w->solver, a, b, rA, rB, fparam3[3 * k], fparam3[3 * k + 1], fparam3[3 * k + 2]);
        else if (ftype[k] == 2)
            new Spring(&w->solver, a, b, rA, rB, fparam3[3 * k], fparam3[3 * k + 1]);
        else
            new IgnoreCollision(&w->solver, a, b);
    }
    w->solver.world.syncFromLegacy(w->solver);
    rebuild_index(w);
    return w;
}

void *ref_create(const RefParams *params, int nBodies, const float *size3, const float *density,
                 const float *friction, const float *pos3, const float *vel3, const float *quat4, int nForces,
                 const int *ftype, const int *fa, const int *fb, const float *frA3, const float *frB3,
                 const float *fparam3)
{
    return ref_create_shapes(params, nBodies, nullptr, nullptr, size3, density, friction, pos3, vel3, quat4, nForces,
                             ftype, fa, fb, frA3, frB3, fparam3);
}

void ref_destroy(void *p) { delete (RefWorld *)p; }

void ref_set_params(void *p, const RefParams *params) { apply_params(((RefWorld *)p)->solver, params); }

int ref_step(void *p, int nsteps)
{
    RefWorld *w = (RefWorld *)p;
    for (int s = 0; s < nsteps; ++s)
        w->solver.step();
    return 0;
}

/* Joint edits between steps with the reference's own constructor / fields / destructor
 * (SimulationHost::beginDrag / updateDrag / releaseDrag, simulation_host.cpp:242-274).
 * The handle is the joint's index among the joints added this way. */
int64_t ref_add_joint(void *p, int a, int b, const float *rA3, const float *rB3, float stiffLin, float stiffAng,
                      float fracture)
{
    RefWorld *w = (RefWorld *)p;
    Rigid *A = a >= 0 ? w->list[a] : 0;
    Joint *j = new Joint(&w->solver, A, w->list[b], float3{rA3[0], rA3[1], rA3[2]}, float3{rB3[0], rB3[1], rB3[2]},
                         stiffLin, stiffAng, fracture);
    w->solver.world.syncFromLegacy(w->solver);
    w->added.push_back(j);
    return (int64_t)w->added.size() - 1;
}

int ref_set_joint_anchor(void *p, int64_t handle, const float *rA3)
{
    RefWorld *w = (RefWorld *)p;
    if (handle < 0 || handle >= (int64_t)w->added.size() || !w->added[handle])
        return -1;
    w->added[handle]->rA = float3{rA3[0], rA3[1], rA3[2]};
    return 0;
}

int ref_remove_joint(void *p, int64_t handle)
{
    RefWorld *w = (RefWorld *)p;
    if (handle < 0 || handle >= (int64_t)w->added.size() || !w->added[handle])
        return -1;
    delete w->added[handle];
    w->added[handle] = 0;
    w->solver.world.syncFromLegacy(w->solver);
    return 0;
}

/* The dense SimWorld bodies, the source of the viewer bridge's snapshots
 * (viewer_bridge.cpp:748-842), synced from the objects as finishStep does; listIndex maps a
 * dense id to its body's list index (-1 for an inactive slot). Returns the slot count. */
int ref_world_bodies(void *p, int *active, int *shape, float *mass, float *pos3, float *quat4, float *size3,
                     float *radius, float *halfLength, int *listIndex)
{
    RefWorld *w = (RefWorld *)p;
    w->solver.world.syncFromLegacy(w->solver);
    const SimWorld &sw = w->solver.world;
    int n = (int)sw.bodies.size();
    if (!active)
        return n;
    for (int i = 0; i < n; ++i)
    {
        const SimBodyData &b = sw.bodies[i];
        active[i] = b.active ? 1 : 0;
        shape[i] = (int)b.shape.type;
        mass[i] = b.mass;
        pos3[3 * i] = b.positionLin.x;
        pos3[3 * i + 1] = b.positionLin.y;
        pos3[3 * i + 2] = b.positionLin.z;
        quat4[4 * i] = b.positionAng.x;
        quat4[4 * i + 1] = b.positionAng.y;
        quat4[4 * i + 2] = b.positionAng.z;
        quat4[4 * i + 3] = b.positionAng.w;
        size3[3 * i] = b.shape.size.x;
        size3[3 * i + 1] = b.shape.size.y;
        size3[3 * i + 2] = b.shape.size.z;
        radius[i] = b.shape.radius;
        halfLength[i] = b.shape.halfLength;
        auto it = b.source ? w->index.find(b.source) : w->index.end();
        listIndex[i] = it == w->index.end() ? -1 : it->second;
    }
    return n;
}

int ref_broadphase_only(void *p)
{
    RefWorld *w = (RefWorld *)p;
    w->solver.benchmarkBroadphaseOnly();
    return 0;
}

int ref_prepare(void *p)
{
    ((RefWorld *)p)->solver.prepareStep();
    return 0;
}

/* prepareStep with the broadphase replaced by the given pairs and the narrowphase of the
 * given entries' pairs by their contacts, exactly as stepCpuReferenceWithExternalBroadphase
 * (solver.cpp:949-957) sets them up around stepCpuReference; the external state is only read
 * by prepareStep (broadphaseExternalPairs, Manifold::initialize), so it is cleared right after.
 * Bodies are list indices (mapped to the reference's dense ids here); contacts use the
 * ref_get_manifolds layout. */
int ref_prepare_external(void *p, int nPairs, const int *ab2, int nEntries, const int *eab2, const int *num,
                         const float *basis9, const int *keys8, const float *contact15x8, const int *stick8)
{
    RefWorld *w = (RefWorld *)p;
    Solver &s = w->solver;
    auto dense = [&](int i) -> BodyId {
        return (i >= 0 && i < (int)w->list.size()) ? w->list[i]->denseId : INVALID_BODY_ID;
    };
    std::vector<BroadphasePair> pairs;
    for (int k = 0; k < nPairs; ++k)
        pairs.push_back(BroadphasePair{dense(ab2[2 * k]), dense(ab2[2 * k + 1])});
    std::vector<ExternalManifoldContact> contacts((size_t)nEntries);
    for (int e = 0; e < nEntries; ++e)
    {
        ExternalManifoldContact &c = contacts[e];
        c = ExternalManifoldContact{};
        c.bodyA = dense(eab2[2 * e]);
        c.bodyB = dense(eab2[2 * e + 1]);
        c.numContacts = num[e];
        std::memcpy(&c.basis, basis9 + 9 * e, 36);
        for (int i = 0; i < 8; ++i)
        {
            Manifold::Contact &m = c.contacts[i];
            const float *v = contact15x8 + (8 * e + i) * 15;
            m.feature.key = keys8[8 * e + i];
            std::memcpy(&m.rA, v, 12);
            std::memcpy(&m.rB, v + 3, 12);
            std::memcpy(&m.C0, v + 6, 12);
            std::memcpy(&m.penalty, v + 9, 12);
            std::memcpy(&m.lambda, v + 12, 12);
            m.stick = stick8[8 * e + i] != 0;
        }
    }
    s.setExternalManifoldContacts(contacts);
    s.externalBroadphasePairs = pairs;
    s.useExternalBroadphasePairs = true;
    s.prepareStep();
    s.useExternalBroadphasePairs = false;
    s.externalBroadphasePairs.clear();
    s.clearExternalManifoldContacts();
    return 0;
}

int ref_iterate(void *p)
{
    ((RefWorld *)p)->solver.iteratePrimalDualCpu();
    return 0;
}

/* Primal sweep in the given order of list indices (colour order); bodies not listed
 * follow in their original list order (the sweep skips them: static or force-less). */
int ref_iterate_ordered(void *p, const int *order, int count)
{
    RefWorld *w = (RefWorld *)p;
    size_t n = w->list.size();
    std::vector<char> listed(n, 0);
    std::vector<Rigid *> seq;
    seq.reserve(n);
    for (int k = 0; k < count; ++k)
    {
        seq.push_back(w->list[order[k]]);
        listed[order[k]] = 1;
    }
    for (size_t i = 0; i < n; ++i)
        if (!listed[i])
            seq.push_back(w->list[i]);
    for (size_t i = 0; i < seq.size(); ++i)
        seq[i]->next = i + 1 < seq.size() ? seq[i + 1] : 0;
    w->solver.bodies = seq.empty() ? 0 : seq[0];
    w->solver.iteratePrimalDualCpu();
    for (size_t i = 0; i < n; ++i)
        w->list[i]->next = i + 1 < n ? w->list[i + 1] : 0;
    w->solver.bodies = n ? w->list[0] : 0;
    return 0;
}

int ref_finish(void *p)
{
    ((RefWorld *)p)->solver.finishStep();
    return 0;
}

int ref_num_bodies(void *p) { return (int)((RefWorld *)p)->list.size(); }

void ref_get_bodies(void *p, float *pos3, float *quat4, float *vel3, float *angvel3, float *prevvel3)
{
    RefWorld *w = (RefWorld *)p;
    for (size_t i = 0; i < w->list.size(); ++i)
    {
        const Rigid *b = w->list[i];
        if (pos3)
            std::memcpy(pos3 + 3 * i, &b->positionLin, 12);
        if (quat4)
            std::memcpy(quat4 + 4 * i, &b->positionAng, 16);
        if (vel3)
            std::memcpy(vel3 + 3 * i, &b->velocityLin, 12);
        if (angvel3)
            std::memcpy(angvel3 + 3 * i, &b->velocityAng, 12);
        if (prevvel3)
            std::memcpy(prevvel3 + 3 * i, &b->prevVelocityLin, 12);
    }
}

void ref_get_body_props(void *p, float *mass, float *moment3, float *radius, float *size3, float *friction)
{
    RefWorld *w = (RefWorld *)p;
    for (size_t i = 0; i < w->list.size(); ++i)
    {
        const Rigid *b = w->list[i];
        if (mass)
            mass[i] = b->mass;
        if (moment3)
            std::memcpy(moment3 + 3 * i, &b->moment, 12);
        if (radius)
            radius[i] = b->radius;
        if (size3)
            std::memcpy(size3 + 3 * i, &b->size, 12);
        if (friction)
            friction[i] = b->friction;
    }
}

int ref_num_manifolds(void *p)
{
    return (int)forces_of_type<Manifold>((RefWorld *)p, SIM_CONSTRAINT_MANIFOLD).size();
}

/* Same layout as oracle_get_manifolds; seq is the creation rank among live manifolds. */
void ref_get_manifolds(void *p, int *ab2, int64_t *seq, int *ncontacts, float *basis9, float *friction, int *keys8,
                       float *contact15x8, int *stick8)
{
    RefWorld *w = (RefWorld *)p;
    std::vector<Manifold *> ms = forces_of_type<Manifold>(w, SIM_CONSTRAINT_MANIFOLD);
    for (size_t i = 0; i < ms.size(); ++i)
    {
        const Manifold *m = ms[i];
        if (ab2)
        {
            ab2[2 * i] = w->index[m->bodyA];
            ab2[2 * i + 1] = w->index[m->bodyB];
        }
        if (seq)
            seq[i] = (int64_t)i;
        if (ncontacts)
            ncontacts[i] = m->numContacts;
        if (basis9)
            std::memcpy(basis9 + 9 * i, &m->basis, 36);
        if (friction)
            friction[i] = m->friction;
        for (int k = 0; k < 8; ++k)
        {
            const Manifold::Contact &c = m->contacts[k];
            bool live = k < m->numContacts;
            if (keys8)
                keys8[8 * i + k] = live ? c.feature.key : 0;
            if (stick8)
                stick8[8 * i + k] = live ? (int)c.stick : 0;
            if (contact15x8)
            {
                float *o = contact15x8 + (8 * i + k) * 15;
                if (live)
                {
                    std::memcpy(o, &c.rA, 12);
                    std::memcpy(o + 3, &c.rB, 12);
                    std::memcpy(o + 6, &c.C0, 12);
                    std::memcpy(o + 9, &c.penalty, 12);
                    std::memcpy(o + 12, &c.lambda, 12);
                }
                else
                    std::memset(o, 0, 60);
            }
        }
    }
}

int ref_num_joints(void *p) { return (int)forces_of_type<Joint>((RefWorld *)p, SIM_CONSTRAINT_JOINT).size(); }

void ref_get_joints(void *p, int *ab2, float *state18, int *broken)
{
    RefWorld *w = (RefWorld *)p;
    std::vector<Joint *> js = forces_of_type<Joint>(w, SIM_CONSTRAINT_JOINT);
    for (size_t i = 0; i < js.size(); ++i)
    {
        const Joint *j = js[i];
        if (ab2)
        {
            ab2[2 * i] = j->bodyA ? w->index[j->bodyA] : -1;
            ab2[2 * i + 1] = w->index[j->bodyB];
        }
        if (state18)
        {
            float *o = state18 + 18 * i;
            std::memcpy(o, &j->C0Lin, 12);
            std::memcpy(o + 3, &j->C0Ang, 12);
            std::memcpy(o + 6, &j->penaltyLin, 12);
            std::memcpy(o + 9, &j->penaltyAng, 12);
            std::memcpy(o + 12, &j->lambdaLin, 12);
            std::memcpy(o + 15, &j->lambdaAng, 12);
        }
        if (broken)
            broken[i] = j->broken ? 1 : 0;
    }
}

/* [0] pair checks, [1] sphere hits, [2] constrained hits, [3] manifolds created,
 * [4] manifolds alive, [5] contacts alive, [6] primal force visits, [7] -, [8] - */
void ref_get_counters(void *p, int64_t *out9)
{
    RefWorld *w = (RefWorld *)p;
    const SolverStats &s = w->solver.stats;
    out9[0] = s.pairChecks;
    out9[1] = s.sphereHits;
    out9[2] = s.constrainedHits;
    out9[3] = s.manifoldsCreated;
    out9[4] = s.manifoldCount;
    int64_t contacts = 0;
    for (Force *f = w->solver.forces; f != 0; f = f->next)
        if (f->type == SIM_CONSTRAINT_MANIFOLD)
            contacts += ((Manifold *)f)->numContacts;
    out9[5] = contacts;
    out9[6] = s.primalForceVisits;
    out9[7] = 0;
    out9[8] = 0;
}

/* Manifold::collide on two free-standing boxes (collide.cpp:1154-1181 -> collideBoxes). */
int ref_collide_boxes(const float *posA3, const float *quatA4, const float *sizeA3, const float *posB3,
                      const float *quatB4, const float *sizeB3, int *keys8, float *rA3x8, float *rB3x8, float *basis9)
{
    Solver s;
    Rigid *a = new Rigid(&s, float3{sizeA3[0], sizeA3[1], sizeA3[2]}, 1.0f, 0.5f, float3{posA3[0], posA3[1], posA3[2]});
    Rigid *b = new Rigid(&s, float3{sizeB3[0], sizeB3[1], sizeB3[2]}, 1.0f, 0.5f, float3{posB3[0], posB3[1], posB3[2]});
    a->positionAng = quat{quatA4[0], quatA4[1], quatA4[2], quatA4[3]};
    b->positionAng = quat{quatB4[0], quatB4[1], quatB4[2], quatB4[3]};
    Manifold::Contact contacts[8] = {};
    float3x3 basis = {};
    int n = Manifold::collide(a, b, contacts, basis);
    for (int i = 0; i < 8; ++i)
    {
        keys8[i] = i < n ? contacts[i].feature.key : 0;
        float3 z = {0, 0, 0};
        std::memcpy(rA3x8 + 3 * i, i < n ? &contacts[i].rA : &z, 12);
        std::memcpy(rB3x8 + 3 * i, i < n ? &contacts[i].rB : &z, 12);
    }
    std::memcpy(basis9, &basis, 36);
    return n;
}

} // extern "C"
