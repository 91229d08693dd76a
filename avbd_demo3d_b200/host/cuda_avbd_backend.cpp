// CUDA AVBD physics backend for the reference solver: the reference-side binding of the
// C ABI (include/avbd_cuda.h). See cuda_avbd_backend.h.
//
// step(Solver&) keeps the reference's object graph as the source of truth at step
// boundaries, as the WebGPU lane does (avbd_gpu_solver.cpp:2110-2185):
//   1. if the bodies or forces changed since the last step (scene load, drag joint,
//      mesh import), upload the whole world; otherwise push only body state;
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
        if (!loaded_ || topologyChanged(solver))
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

  private:
    AvbdContext *ctx_ = nullptr;
    bool failed_ = false;
    bool loaded_ = false;
    std::vector<Rigid *> bodies_; // list order at upload
    std::unordered_map<const Rigid *, int> index_;
    std::vector<Force *> forcesSeen_; // solver.forces after the last mirror, newest first
    std::unordered_map<int64_t, Force *> bySeq_;

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
        return s.broadphaseMode == BROADPHASE_ALL_PAIRS ? AVBD_BROADPHASE_ALL_PAIRS : AVBD_BROADPHASE_GRID;
    }

    bool checkShapes(Solver &solver)
    {
        for (Rigid *b = solver.bodies; b; b = b->next)
            if (b->shape.type != RIGID_SHAPE_BOX)
            {
                std::fprintf(stderr, "CUDA AVBD backend: only box bodies are supported\n");
                failed_ = true;
                return false;
            }
        if (solver.broadphaseMode == BROADPHASE_SWEEP_AND_PRUNE)
        {
            std::fprintf(stderr, "CUDA AVBD backend: sweep-and-prune broadphase is not available on the GPU\n");
            failed_ = true;
            return false;
        }
        return true;
    }

    bool topologyChanged(Solver &solver)
    {
        size_t i = 0;
        for (Rigid *b = solver.bodies; b; b = b->next, ++i)
            if (i >= bodies_.size() || bodies_[i] != b)
                return true;
        if (i != bodies_.size())
            return true;
        i = 0;
        for (Force *f = solver.forces; f; f = f->next, ++i)
            if (i >= forcesSeen_.size() || forcesSeen_[i] != f)
                return true;
        return i != forcesSeen_.size();
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
        std::vector<float> pos, quat, vel, ang, prev, size, mass, moment, friction, radius;
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
        }
    }

    static AvbdBodies view(int n, const BodyArrays &a)
    {
        return AvbdBodies{n,         a.pos.data(),    a.quat.data(),   a.vel.data(),      a.ang.data(),
                          a.prev.data(), a.size.data(), a.mass.data(), a.moment.data(), a.friction.data(),
                          a.radius.data()};
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
                const float3 *v[] = {&j->rA, &j->rB, &j->C0Lin, &j->C0Ang, &j->penaltyLin, &j->penaltyAng,
                                     &j->lambdaLin, &j->lambdaAng};
                for (const float3 *x : v)
                {
                    jst.push_back(x->x);
                    jst.push_back(x->y);
                    jst.push_back(x->z);
                }
                jst.push_back(j->stiffnessLin);
                jst.push_back(j->stiffnessAng);
                jst.push_back(j->fracture);
                jst.push_back(j->torqueArm);
                jbroken.push_back(j->broken ? 1 : 0);
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

        forcesSeen_.clear();
        for (Force *f = solver.forces; f; f = f->next)
            forcesSeen_.push_back(f);

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
