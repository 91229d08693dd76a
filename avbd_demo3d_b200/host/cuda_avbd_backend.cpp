// CUDA AVBD physics backend for the reference solver: the reference-side binding of the
// C ABI (include/avbd_cuda.h). See cuda_avbd_backend.h.
//
// step(Solver&) keeps the reference's object graph as the source of truth at step
// boundaries, as the WebGPU lane does (avbd_gpu_solver.cpp:2110-2185):
//   1. if the body list changed since the last step (scene load, mesh import), upload the
//      whole world. Otherwise diff the force list against the one mirrored after the last
//      step: joints created, deleted or edited between steps (SimulationHost's drag,
//      simulation_host.cpp:242-274) go to the device as joint edits; any other change of
//      forces reloads the world; body state is pushed every step;
//   2. run Solver::step's work on the GPU (avbd_step);
//   3. write bodies back, mirror created/removed manifolds and removed joints into the
//      object graph in the device's creation order, copy contact and joint state, and
//      re-sync the dense SimWorld (finishStep, solver.cpp:1296).
// There is no CPU fallback: a failure is reported and the backend stops stepping.
#include "cuda_avbd_backend.h"

#include "avbd_cuda.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace
{

class CudaAvbdBackend : public PhysicsBackend
{
  public:
    explicit CudaAvbdBackend(int device)
    {
        if (avbd_create(&ctx_, device, nullptr) != AVBD_OK)
        {
            std::fprintf(stderr, "CUDA AVBD backend: no CUDA device %d\n", device);
            ctx_ = nullptr;
            failed_ = true;
        }
    }
    ~CudaAvbdBackend() override { avbd_destroy(ctx_); }

    const char *name() const override { return avbd_backend_name(); }

    void step(Solver &solver) override
    {
        if (failed_)
            return;
        if (!checkShapes(solver))
            return;
        int sync = loaded_ && !bodiesChanged(solver) ? syncForces(solver) : SYNC_RELOAD;
        if (sync == SYNC_FAILED)
            return;
        if (sync == SYNC_RELOAD)
        {
            if (!upload(solver))
                return;
        }
        else if (!pushBodyState(solver))
            return;
        AvbdParams p{solver.dt,    solver.gravity, solver.iterations, solver.alpha, solver.betaLin,
                     solver.betaAng, solver.gamma, broadphaseOf(solver)};
        if (!ok(avbd_set_params(ctx_, &p), "avbd_set_params") || !ok(avbd_step(ctx_, 1), "avbd_step"))
            return;
        readBack(solver);
    }

    AvbdContext *context() const { return ctx_; }
    int uploads() const { return uploads_; }
    int jointEdits() const { return jointEdits_; }

  private:
    AvbdContext *ctx_ = nullptr;
    bool failed_ = false;
    bool loaded_ = false;
    int uploads_ = 0, jointEdits_ = 0;
    std::vector<Rigid *> bodies_; // list order at upload
    std::unordered_map<const Rigid *, int> index_;
    std::unordered_map<int64_t, Force *> bySeq_;

    // solver.forces as mirrored after the last step, newest first, with what a later diff
    // compares: type, bodies and (joints) the 28-float state the device holds
    struct Seen
    {
        Force *f;
        int64_t seq;
        int type;
        const Rigid *a, *b;
        float st[28];
        int32_t broken;
    };
    std::vector<Seen> seen_;
    enum
    {
        SYNC_DONE = 0,
        SYNC_RELOAD = 1,
        SYNC_FAILED = 2
    };

    bool ok(int rc, const char *what)
    {
        if (rc == AVBD_OK)
            return true;
        std::fprintf(stderr, "CUDA AVBD backend: %s failed (%d): %s\n", what, rc, avbd_last_error(ctx_));
        failed_ = true;
        return false;
    }

    static int32_t broadphaseOf(const Solver &s)
    {
        return s.broadphaseMode == BROADPHASE_ALL_PAIRS       ? AVBD_BROADPHASE_ALL_PAIRS
               : s.broadphaseMode == BROADPHASE_SWEEP_AND_PRUNE ? AVBD_BROADPHASE_SAP
                                                                : AVBD_BROADPHASE_GRID;
    }

    bool checkShapes(Solver &solver)
    {
        for (Rigid *b = solver.bodies; b; b = b->next)
            if (b->shape.type < RIGID_SHAPE_BOX || b->shape.type > RIGID_SHAPE_CYLINDER)
            {
                std::fprintf(stderr, "CUDA AVBD backend: unknown body shape %d\n", (int)b->shape.type);
                failed_ = true;
                return false;
            }
        return true;
    }

    bool bodiesChanged(Solver &solver) const
    {
        size_t i = 0;
        for (Rigid *b = solver.bodies; b; b = b->next, ++i)
            if (i >= bodies_.size() || bodies_[i] != b)
                return true;
        return i != bodies_.size();
    }

    static void jointState(const Joint *j, float *st, int32_t *broken)
    {
        const float3 *v[] = {&j->rA,         &j->rB,         &j->C0Lin,     &j->C0Ang,
                             &j->penaltyLin, &j->penaltyAng, &j->lambdaLin, &j->lambdaAng};
        for (int k = 0; k < 8; ++k)
        {
            st[3 * k] = v[k]->x;
            st[3 * k + 1] = v[k]->y;
            st[3 * k + 2] = v[k]->z;
        }
        st[24] = j->stiffnessLin;
        st[25] = j->stiffnessAng;
        st[26] = j->fracture;
        st[27] = j->torqueArm;
        *broken = j->broken ? 1 : 0;
    }

    // Diff solver.forces against seen_. The reference only ever prepends a new force
    // (force.cpp:17-22) and unlinks a deleted one, so the survivors keep their order: a walk
    // from the oldest end matches them, and what is left at the head is new. A new force
    // that reuses a deleted one's address and is matched in its place keeps the same order
    // relative to every survivor, and differs in type, bodies or state, which the checks
    // below see. Joint creation, deletion and edits become device edits; anything else
    // asks for a reload.
    int syncForces(Solver &solver)
    {
        std::vector<Force *> cur;
        for (Force *f = solver.forces; f; f = f->next)
            cur.push_back(f);
        std::vector<long> match(seen_.size(), -1);
        long i = (long)cur.size() - 1;
        for (long k = (long)seen_.size() - 1; k >= 0 && i >= 0; --k)
            if (cur[(size_t)i] == seen_[(size_t)k].f)
                match[(size_t)k] = i--;
        long fresh = i + 1; // cur[0, fresh) were created since the last step

        std::vector<int64_t> removed;
        std::vector<int32_t> wab;
        std::vector<int64_t> wseq;
        std::vector<float> wst;
        std::vector<int32_t> wbroken;
        float st[28];
        int32_t broken;
        for (size_t k = 0; k < seen_.size(); ++k)
        {
            const Seen &s = seen_[k];
            if (s.seq < 0)
                return SYNC_RELOAD;
            if (match[k] < 0)
            {
                if (s.type != SIM_CONSTRAINT_JOINT)
                    return SYNC_RELOAD;
                removed.push_back(s.seq);
                continue;
            }
            Force *f = cur[(size_t)match[k]];
            if (f->type != s.type || f->bodyA != s.a || f->bodyB != s.b)
                return SYNC_RELOAD;
            if (f->type != SIM_CONSTRAINT_JOINT)
                continue;
            jointState((Joint *)f, st, &broken);
            if (std::memcmp(st, s.st, sizeof(st)) != 0 || broken != s.broken)
            {
                wab.push_back(indexOf(f->bodyA));
                wab.push_back(indexOf(f->bodyB));
                wseq.push_back(s.seq);
                wst.insert(wst.end(), st, st + 28);
                wbroken.push_back(broken);
            }
        }
        std::vector<Joint *> added;
        std::vector<int32_t> aab;
        std::vector<float> ast;
        std::vector<int32_t> abroken;
        for (long c = fresh - 1; c >= 0; --c) // creation order
        {
            Force *f = cur[(size_t)c];
            if (f->type != SIM_CONSTRAINT_JOINT || indexOf(f->bodyB) < 0 || (f->bodyA && indexOf(f->bodyA) < 0))
                return SYNC_RELOAD;
            added.push_back((Joint *)f);
            aab.push_back(indexOf(f->bodyA));
            aab.push_back(indexOf(f->bodyB));
            jointState((Joint *)f, st, &broken);
            ast.insert(ast.end(), st, st + 28);
            abroken.push_back(broken);
        }
        if (!removed.empty())
        {
            if (!ok(avbd_remove_joints(ctx_, (int32_t)removed.size(), removed.data()), "avbd_remove_joints"))
                return SYNC_FAILED;
            jointEdits_++;
            for (int64_t s : removed)
                bySeq_.erase(s); // the caller deleted the object
        }
        if (!added.empty())
        {
            int64_t next = 0;
            if (!ok(avbd_next_seq(ctx_, &next), "avbd_next_seq"))
                return SYNC_FAILED;
            std::vector<int64_t> aseq(added.size());
            for (size_t a = 0; a < added.size(); ++a)
            {
                aseq[a] = next + (int64_t)a;
                bySeq_[aseq[a]] = added[a];
            }
            AvbdJoints jv{(int32_t)added.size(), aab.data(), aseq.data(), ast.data(), abroken.data()};
            if (!ok(avbd_add_joints(ctx_, &jv), "avbd_add_joints"))
                return SYNC_FAILED;
            jointEdits_++;
        }
        if (!wseq.empty())
        {
            AvbdJoints jv{(int32_t)wseq.size(), wab.data(), wseq.data(), wst.data(), wbroken.data()};
            if (!ok(avbd_write_joints(ctx_, &jv), "avbd_write_joints"))
                return SYNC_FAILED;
            jointEdits_++;
        }
        return SYNC_DONE;
    }

    int indexOf(const Rigid *b) const
    {
        if (!b)
            return -1;
        auto it = index_.find(b);
        return it == index_.end() ? -1 : it->second;
    }

    struct BodyArrays
    {
        std::vector<float> pos, quat, vel, ang, prev, size, mass, moment, friction, radius, shapeRadius, halfLength;
        std::vector<int32_t> shape;
    };

    void gatherBodies(BodyArrays &a) const
    {
        size_t n = bodies_.size();
        a.pos.resize(3 * n);
        a.quat.resize(4 * n);
        a.vel.resize(3 * n);
        a.ang.resize(3 * n);
        a.prev.resize(3 * n);
        a.size.resize(3 * n);
        a.mass.resize(n);
        a.moment.resize(3 * n);
        a.friction.resize(n);
        a.radius.resize(n);
        a.shape.resize(n);
        a.shapeRadius.resize(n);
        a.halfLength.resize(n);
        for (size_t i = 0; i < n; ++i)
        {
            const Rigid *b = bodies_[i];
            std::memcpy(&a.pos[3 * i], &b->positionLin, 12);
            std::memcpy(&a.quat[4 * i], &b->positionAng, 16);
            std::memcpy(&a.vel[3 * i], &b->velocityLin, 12);
            std::memcpy(&a.ang[3 * i], &b->velocityAng, 12);
            std::memcpy(&a.prev[3 * i], &b->prevVelocityLin, 12);
            std::memcpy(&a.size[3 * i], &b->size, 12);
            a.mass[i] = b->mass;
            std::memcpy(&a.moment[3 * i], &b->moment, 12);
            a.friction[i] = b->friction;
            a.radius[i] = b->radius;
            a.shape[i] = (int32_t)b->shape.type; // RigidShapeType values are the ABI's AVBD_SHAPE_*
            a.shapeRadius[i] = b->shape.radius;
            a.halfLength[i] = b->shape.halfLength;
        }
    }

    static AvbdBodies view(int n, const BodyArrays &a)
    {
        return AvbdBodies{n,
                          a.pos.data(),
                          a.quat.data(),
                          a.vel.data(),
                          a.ang.data(),
                          a.prev.data(),
                          a.size.data(),
                          a.mass.data(),
                          a.moment.data(),
                          a.friction.data(),
                          a.radius.data(),
                          a.shape.data(),
                          a.shapeRadius.data(),
                          a.halfLength.data()};
    }

    bool pushBodyState(Solver &)
    {
        BodyArrays a;
        gatherBodies(a);
        AvbdBodies v = view((int)bodies_.size(), a);
        return ok(avbd_write_bodies(ctx_, &v), "avbd_write_bodies");
    }

    bool upload(Solver &solver)
    {
        bodies_.clear();
        index_.clear();
        for (Rigid *b = solver.bodies; b; b = b->next)
        {
            index_[b] = (int)bodies_.size();
            bodies_.push_back(b);
        }
        BodyArrays a;
        gatherBodies(a);

        // sequence number = creation rank (solver.forces is newest first, force.cpp:17-22)
        std::vector<Force *> forces;
        for (Force *f = solver.forces; f; f = f->next)
            forces.push_back(f);
        int64_t total = (int64_t)forces.size();
        std::vector<int32_t> jab, sab, iab, mab, jbroken, mn, mkeys, mstick;
        std::vector<int64_t> jseq, sseq, iseq, mseq;
        std::vector<float> jst, sst, mbasis, mfric, mcontact;
        bySeq_.clear();
        for (int64_t k = total - 1; k >= 0; --k) // creation order
        {
            Force *f = forces[(size_t)k];
            int64_t seq = total - 1 - k;
            bySeq_[seq] = f;
            int a0 = indexOf(f->bodyA), b0 = indexOf(f->bodyB);
            if (f->type == SIM_CONSTRAINT_JOINT)
            {
                Joint *j = (Joint *)f;
                jab.push_back(a0);
                jab.push_back(b0);
                jseq.push_back(seq);
                float st[28];
                int32_t broken;
                jointState(j, st, &broken);
                jst.insert(jst.end(), st, st + 28);
                jbroken.push_back(broken);
            }
            else if (f->type == SIM_CONSTRAINT_SPRING)
            {
                Spring *s = (Spring *)f;
                sab.push_back(a0);
                sab.push_back(b0);
                sseq.push_back(seq);
                const float v[8] = {s->rA.x, s->rA.y, s->rA.z, s->rB.x, s->rB.y, s->rB.z, s->rest, s->stiffness};
                sst.insert(sst.end(), v, v + 8);
            }
            else if (f->type == SIM_CONSTRAINT_IGNORE_COLLISION)
            {
                iab.push_back(a0);
                iab.push_back(b0);
                iseq.push_back(seq);
            }
            else if (f->type == SIM_CONSTRAINT_MANIFOLD)
            {
                Manifold *m = (Manifold *)f;
                mab.push_back(a0);
                mab.push_back(b0);
                mseq.push_back(seq);
                mn.push_back(m->numContacts);
                for (int r = 0; r < 3; ++r)
                {
                    mbasis.push_back(m->basis[r].x);
                    mbasis.push_back(m->basis[r].y);
                    mbasis.push_back(m->basis[r].z);
                }
                mfric.push_back(m->friction);
                for (int c = 0; c < 8; ++c)
                {
                    const Manifold::Contact &ct = m->contacts[c];
                    mkeys.push_back(ct.feature.key);
                    mstick.push_back(ct.stick ? 1 : 0);
                    const float3 *v[] = {&ct.rA, &ct.rB, &ct.C0, &ct.penalty, &ct.lambda};
                    for (const float3 *x : v)
                    {
                        mcontact.push_back(x->x);
                        mcontact.push_back(x->y);
                        mcontact.push_back(x->z);
                    }
                }
            }
        }
        AvbdBodies bv = view((int)bodies_.size(), a);
        AvbdJoints jv{(int32_t)jseq.size(), jab.data(), jseq.data(), jst.data(), jbroken.data()};
        AvbdSprings sv{(int32_t)sseq.size(), sab.data(), sseq.data(), sst.data()};
        AvbdIgnores iv{(int32_t)iseq.size(), iab.data(), iseq.data()};
        AvbdManifolds mv{(int32_t)mseq.size(), mab.data(), mseq.data(), mn.data(), mbasis.data(), mfric.data(),
                         mkeys.data(), mcontact.data(), mstick.data()};
        if (!ok(avbd_load_world(ctx_, &bv, &jv, &sv, &iv, &mv, total), "avbd_load_world"))
            return false;
        loaded_ = true;
        uploads_++;
        return true;
    }

    void readBack(Solver &solver)
    {
        int n = (int)bodies_.size();
        std::vector<float> pos(3 * n), quat(4 * n), vel(3 * n), ang(3 * n), prev(3 * n), il(3 * n), ia(4 * n),
            nl(3 * n), na(4 * n);
        AvbdBodyState st{pos.data(), quat.data(), vel.data(), ang.data(), prev.data(),
                         il.data(),  ia.data(),   nl.data(),  na.data()};
        if (!ok(avbd_read_bodies(ctx_, &st), "avbd_read_bodies"))
            return;
        for (int i = 0; i < n; ++i)
        {
            Rigid *b = bodies_[i];
            std::memcpy(&b->positionLin, &pos[3 * i], 12);
            std::memcpy(&b->positionAng, &quat[4 * i], 16);
            std::memcpy(&b->velocityLin, &vel[3 * i], 12);
            std::memcpy(&b->velocityAng, &ang[3 * i], 12);
            std::memcpy(&b->prevVelocityLin, &prev[3 * i], 12);
            std::memcpy(&b->initialLin, &il[3 * i], 12);
            std::memcpy(&b->initialAng, &ia[4 * i], 16);
            std::memcpy(&b->inertialLin, &nl[3 * i], 12);
            std::memcpy(&b->inertialAng, &na[4 * i], 16);
        }

        int32_t M = 0, J = 0;
        if (!ok(avbd_num_manifolds(ctx_, &M), "avbd_num_manifolds") || !ok(avbd_num_joints(ctx_, &J), "avbd_num_joints"))
            return;
        std::vector<int32_t> mab(2 * (size_t)M), mn(M), mkeys(8 * (size_t)M), mstick(8 * (size_t)M);
        std::vector<int64_t> mseq(M);
        std::vector<float> mbasis(9 * (size_t)M), mfric(M), mcontact(120 * (size_t)M);
        AvbdManifoldsOut mo{mab.data(),  mseq.data(),  mn.data(),       mbasis.data(),
                            mfric.data(), mkeys.data(), mcontact.data(), mstick.data()};
        std::vector<int32_t> jab(2 * (size_t)J), jbroken(J);
        std::vector<int64_t> jseq(J);
        std::vector<float> jst(28 * (size_t)J);
        AvbdJointsOut jo{jab.data(), jseq.data(), jst.data(), jbroken.data()};
        if ((M && !ok(avbd_read_manifolds(ctx_, &mo), "avbd_read_manifolds")) ||
            (J && !ok(avbd_read_joints(ctx_, &jo), "avbd_read_joints")))
            return;

        // forces the device no longer has: manifolds without contacts, joints removed
        // after fracture (prepareStep deletes both, solver.cpp:1124-1130)
        std::unordered_map<int64_t, int> live;
        for (int m = 0; m < M; ++m)
            live[mseq[m]] = m;
        for (int j = 0; j < J; ++j)
            live[jseq[j]] = -1 - j;
        std::vector<int64_t> gone;
        for (auto &kv : bySeq_)
        {
            Force *f = kv.second;
            bool tracked = f->type == SIM_CONSTRAINT_MANIFOLD || f->type == SIM_CONSTRAINT_JOINT;
            if (tracked && !live.count(kv.first))
                gone.push_back(kv.first);
        }
        for (int64_t s : gone)
        {
            delete bySeq_[s];
            bySeq_.erase(s);
        }
        // manifolds: create the device's new ones in creation order, copy contact state
        for (int m = 0; m < M; ++m)
        {
            auto it = bySeq_.find(mseq[m]);
            Manifold *man;
            if (it == bySeq_.end())
            {
                man = new Manifold(&solver, bodies_[mab[2 * m]], bodies_[mab[2 * m + 1]]);
                bySeq_[mseq[m]] = man;
            }
            else
                man = (Manifold *)it->second;
            man->numContacts = mn[m];
            man->friction = mfric[m];
            for (int r = 0; r < 3; ++r)
                man->basis[r] = float3{mbasis[9 * m + 3 * r], mbasis[9 * m + 3 * r + 1], mbasis[9 * m + 3 * r + 2]};
            for (int c = 0; c < 8; ++c)
            {
                Manifold::Contact &ct = man->contacts[c];
                const float *v = &mcontact[((size_t)8 * m + c) * 15];
                ct.feature.key = mkeys[8 * m + c];
                ct.rA = float3{v[0], v[1], v[2]};
                ct.rB = float3{v[3], v[4], v[5]};
                ct.C0 = float3{v[6], v[7], v[8]};
                ct.penalty = float3{v[9], v[10], v[11]};
                ct.lambda = float3{v[12], v[13], v[14]};
                ct.stick = mstick[8 * m + c] != 0;
            }
        }
        for (int j = 0; j < J; ++j)
        {
            auto it = bySeq_.find(jseq[j]);
            if (it == bySeq_.end())
                continue;
            Joint *jt = (Joint *)it->second;
            const float *v = &jst[28 * (size_t)j];
            jt->C0Lin = float3{v[6], v[7], v[8]};
            jt->C0Ang = float3{v[9], v[10], v[11]};
            jt->penaltyLin = float3{v[12], v[13], v[14]};
            jt->penaltyAng = float3{v[15], v[16], v[17]};
            jt->lambdaLin = float3{v[18], v[19], v[20]};
            jt->lambdaAng = float3{v[21], v[22], v[23]};
            jt->broken = jbroken[j] != 0;
        }

        std::unordered_map<const Force *, int64_t> seqOf;
        for (auto &kv : bySeq_)
            seqOf[kv.second] = kv.first;
        seen_.clear();
        for (Force *f = solver.forces; f; f = f->next)
        {
            Seen s{};
            s.f = f;
            auto it = seqOf.find(f);
            s.seq = it == seqOf.end() ? -1 : it->second;
            s.type = f->type;
            s.a = f->bodyA;
            s.b = f->bodyB;
            if (f->type == SIM_CONSTRAINT_JOINT)
                jointState((Joint *)f, s.st, &s.broken);
            seen_.push_back(s);
        }

        AvbdStats stats{};
        avbd_get_stats(ctx_, &stats);
        solver.stats = SolverStats{};
        solver.stats.bodyCount = (int)stats.body_count;
        for (Rigid *b = solver.bodies; b; b = b->next)
            if (b->mass > 0)
                solver.stats.activeBodyCount++;
        solver.stats.pairChecks = (int)stats.pair_checks;
        solver.stats.sphereHits = (int)stats.sphere_hits;
        solver.stats.constrainedChecks = (int)stats.sphere_hits;
        solver.stats.constrainedHits = (int)stats.constrained_hits;
        solver.stats.manifoldsCreated = (int)stats.manifolds_created;
        solver.stats.manifoldCount = (int)stats.manifold_count;
        solver.stats.jointCount = (int)stats.joint_count;
        solver.stats.springCount = (int)stats.spring_count;
        for (Force *f = solver.forces; f; f = f->next)
        {
            solver.stats.forceCount++;
            if (f->type == SIM_CONSTRAINT_IGNORE_COLLISION)
                solver.stats.ignoreCollisionCount++;
        }
        solver.world.syncFromLegacy(solver);
    }
};

} // namespace

std::unique_ptr<PhysicsBackend> makeCudaAvbdPhysicsBackend(int device)
{
    return std::unique_ptr<PhysicsBackend>(new CudaAvbdBackend(device));
}

AvbdContext *cudaAvbdBackendContext(PhysicsBackend *backend)
{
    CudaAvbdBackend *b = dynamic_cast<CudaAvbdBackend *>(backend);
    return b ? b->context() : nullptr;
}

int cudaAvbdBackendUploads(PhysicsBackend *backend)
{
    CudaAvbdBackend *b = dynamic_cast<CudaAvbdBackend *>(backend);
    return b ? b->uploads() : 0;
}

int cudaAvbdBackendJointEdits(PhysicsBackend *backend)
{
    CudaAvbdBackend *b = dynamic_cast<CudaAvbdBackend *>(backend);
    return b ? b->jointEdits() : 0;
}
