/*
 * Driver around the DOUBLE-PRECISION twin of the reference solver (test infrastructure).
 *
 * oracle/Makefile (target ref64) writes an FP64 copy of the reference's core sources
 * with make_fp64.py and compiles it with this file into oracle/_ref/libavbd_ref64.so.
 * The scene is built through the reference's public constructors (Rigid, Joint, Spring,
 * IgnoreCollision; solver.h:221, 262, 276, 288) from the same single-precision inputs as
 * every other checker (widened exactly to double) and stepped by the stock CPU backend
 * (Solver::step, solver.cpp:934-937) in the reference's own list order. State is read
 * back in list order (index 0 = the solver's body-list head) as doubles.
 *
 * The same source also compiles against the reference's own (single-precision) headers;
 * every field is copied member by member, whatever its width.
 */
#include "solver.h"

#include <cstdint>
#include <vector>

namespace
{
struct Ref64World
{
    Solver solver;
    std::vector<Rigid *> list;
};

struct Ref64Params // the same layout as the other checkers' parameter block
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

float3 vec3(const float *p) { return float3{p[0], p[1], p[2]}; }

void put3(double *o, const float3 &v)
{
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
}
} // namespace

extern "C"
{

void *ref64_create(const Ref64Params *p, int nBodies, const float *size3, const float *density,
                   const float *friction, const float *pos3, const float *vel3, const float *quat4, int nForces,
                   const int *ftype, const int *fa, const int *fb, const float *frA3, const float *frB3,
                   const float *fparam3)
{
    Ref64World *w = new Ref64World();
    Solver &s = w->solver;
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
    std::vector<Rigid *> created;
    created.reserve(nBodies);
    for (int c = 0; c < nBodies; ++c)
    {
        Rigid *r = new Rigid(&s, vec3(size3 + 3 * c), density[c], friction[c], vec3(pos3 + 3 * c), vec3(vel3 + 3 * c));
        r->positionAng = quat{quat4[4 * c], quat4[4 * c + 1], quat4[4 * c + 2], quat4[4 * c + 3]};
        created.push_back(r);
    }
    for (int k = 0; k < nForces; ++k)
    {
        Rigid *a = fa[k] >= 0 ? created[fa[k]] : 0;
        Rigid *b = created[fb[k]];
        if (ftype[k] == 1)
            new Joint(&s, a, b, vec3(frA3 + 3 * k), vec3(frB3 + 3 * k), fparam3[3 * k], fparam3[3 * k + 1],
                      fparam3[3 * k + 2]);
        else if (ftype[k] == 2)
            new Spring(&s, a, b, vec3(frA3 + 3 * k), vec3(frB3 + 3 * k), fparam3[3 * k], fparam3[3 * k + 1]);
        else
            new IgnoreCollision(&s, a, b);
    }
    s.world.syncFromLegacy(s);
    for (Rigid *b = s.bodies; b != 0; b = b->next)
        w->list.push_back(b);
    return w;
}

void ref64_destroy(void *p) { delete (Ref64World *)p; }

int ref64_step(void *p, int nsteps)
{
    Ref64World *w = (Ref64World *)p;
    for (int s = 0; s < nsteps; ++s)
        w->solver.step();
    return 0;
}

int ref64_num_bodies(void *p) { return (int)((Ref64World *)p)->list.size(); }

/* position (3), orientation (x, y, z, w) and velocities (3 each) per body, list order */
void ref64_get_bodies(void *p, double *pos3, double *quat4, double *vel3, double *angvel3)
{
    Ref64World *w = (Ref64World *)p;
    for (size_t i = 0; i < w->list.size(); ++i)
    {
        const Rigid *b = w->list[i];
        if (pos3)
            put3(pos3 + 3 * i, b->positionLin);
        if (quat4)
        {
            quat4[4 * i] = b->positionAng.x;
            quat4[4 * i + 1] = b->positionAng.y;
            quat4[4 * i + 2] = b->positionAng.z;
            quat4[4 * i + 3] = b->positionAng.w;
        }
        if (vel3)
            put3(vel3 + 3 * i, b->velocityLin);
        if (angvel3)
            put3(angvel3 + 3 * i, b->velocityAng);
    }
}

/* 1 when the reference's scalar type is double (this build), 0 for the stock build */
int ref64_is_double(void) { return sizeof(((Rigid *)0)->mass) == sizeof(double) ? 1 : 0; }

} // extern "C"
