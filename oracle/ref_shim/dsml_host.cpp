/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * Host build of the reference's OWN scene-file parser: src/parser.cpp and
 * src/DEMSimulation.cpp, with the rapidxml headers the reference ships in
 * its includes/ directory, are compiled unmodified from the reference tree
 * (paths supplied by oracle/Makefile with -I).  This file only supplies what
 * those sources expect from their surroundings:
 *
 *  - MAIN_CUH is pre-defined so the reference's main.cuh (CUDA/GL state
 *    structs) is skipped, with USE_BIG_PARTICLE 0: the step has no control
 *    particle, and the reference's example scenes without a <controlled>
 *    tag parse only in that configuration;
 *  - the three stream operators functions.cuh declares (defined in the
 *    reference's functions.cu, which is not built here) for
 *    DEMSimulation::printConfiguration;
 *  - C entry points that run the parser's load steps the way
 *    DEMSimulation::loadFromFile does (DEMSimulation.cpp:45-60) but return
 *    the error text instead of calling exit(), and copy the parsed scene out
 *    into flat arrays.
 *
 * Single-threaded: the parsed scene lives in one static object.
 */
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>

typedef unsigned int uint;

#define MAIN_CUH 1
#define USE_BIG_PARTICLE 0
#define USE_ATOMIC 0
#define MAX_PARTICLES_TYPES 10

struct ParticleProperties;
struct ParticlesValues;
struct SystemProperties;
struct RenderParameters;

#include "parser.cpp"
#include "DEMSimulation.cpp"

std::ostream& operator<<(std::ostream& o, const uint2& v) { return o << v.x << "," << v.y; }
std::ostream& operator<<(std::ostream& o, const float2& v) { return o << v.x << "," << v.y; }
std::ostream& operator<<(std::ostream& o, const float3& v) {
    return o << v.x << "," << v.y << "," << v.z;
}

namespace {
DEMSimulation g_sim;
}

extern "C" {

/* Parses `path` as DEMSimulation::loadFromFile does; 0 on success, 1 with
 * the reference's message in err on a parse error. */
int ref_dsml_load(const char* path, char* err, int errlen) {
    g_sim = DEMSimulation();
    try {
        DEMParser parser(path);
        g_sim.parameters = parser.loadParameters();
        g_sim.environment = parser.loadEnvironment();
        g_sim.properties = parser.loadProperties();
        g_sim.particles = parser.loadParticles(&g_sim.properties);
    } catch (std::string msg) {
        snprintf(err, (size_t)errlen, "%s", msg.c_str());
        return 1;
    } catch (const char* msg) {
        snprintf(err, (size_t)errlen, "%s", msg);
        return 1;
    }
    return 0;
}

/* numTypes, numRect, numTri, numSingle, numFollowSingle, numFollowParam,
 * controlledType */
void ref_dsml_counts(int* out) {
    out[0] = (int)g_sim.properties.particleTypes.size();
    out[1] = (int)g_sim.particles.start.size();
    out[2] = (int)g_sim.particles.t_pos.size();
    out[3] = (int)g_sim.particles.pos.size();
    out[4] = (int)g_sim.particles.followedParticles.size();
    out[5] = (int)g_sim.parameters.followedParticles.size();
    out[6] = -1;  // not parsed with USE_BIG_PARTICLE 0
}

/* timeStep, simDuration, imageDIMy, dim x, y, gravity x, y, knWall, ktWall */
void ref_dsml_params(double* out) {
    out[0] = g_sim.parameters.timeStep;
    out[1] = g_sim.parameters.simDuration;
    out[2] = g_sim.parameters.imageDIMy;
    out[3] = g_sim.environment.dimension.x;
    out[4] = g_sim.environment.dimension.y;
    out[5] = g_sim.environment.gravity.x;
    out[6] = g_sim.environment.gravity.y;
    out[7] = g_sim.environment.boundaryNormalStiffness;
    out[8] = g_sim.environment.boundaryShearStiffness;
}

/* mass, radius, kn, kt, cn, eb, mu, at, colour r, g, b */
void ref_dsml_type(int i, double* out, char* id, int idlen) {
    const DEMParticleType& t = g_sim.properties.particleTypes[i];
    const float v[11] = {t.mass, t.radius, t.normalStiffness, t.shearStiffness, t.normalDamping,
                         t.boundaryDamping, t.frictionCoefficient, t.attractCoefficient,
                         t.color.x, t.color.y, t.color.z};
    for (int k = 0; k < 11; ++k) out[k] = v[k];
    snprintf(id, (size_t)idlen, "%s", t.id.c_str());
}

/* start x, y, end x, y, num x, y; its type list */
int ref_dsml_rect(int i, double* out, int* types) {
    const DEMParticles& p = g_sim.particles;
    out[0] = p.start[i].x; out[1] = p.start[i].y;
    out[2] = p.end[i].x;   out[3] = p.end[i].y;
    out[4] = p.num[i].x;   out[5] = p.num[i].y;
    for (size_t k = 0; k < p.types[i].size(); ++k) types[k] = p.types[i][k];
    return (int)p.types[i].size();
}

/* pos x, y, width, num; its type list */
int ref_dsml_tri(int i, double* out, int* types) {
    const DEMParticles& p = g_sim.particles;
    out[0] = p.t_pos[i].x; out[1] = p.t_pos[i].y;
    out[2] = p.width[i];   out[3] = p.t_num[i];
    for (size_t k = 0; k < p.t_types[i].size(); ++k) types[k] = p.t_types[i][k];
    return (int)p.t_types[i].size();
}

/* pos x, y, vel x, y, theta, omega, type */
void ref_dsml_single(int i, double* out) {
    const DEMParticles& p = g_sim.particles;
    out[0] = p.pos[i].x; out[1] = p.pos[i].y;
    out[2] = p.vel[i].x; out[3] = p.vel[i].y;
    out[4] = p.theta[i]; out[5] = p.omega[i];
    out[6] = p.type[i];
}

void ref_dsml_followed(int* singles, int* params) {
    for (size_t k = 0; k < g_sim.particles.followedParticles.size(); ++k)
        singles[k] = g_sim.particles.followedParticles[k];
    for (size_t k = 0; k < g_sim.parameters.followedParticles.size(); ++k)
        params[k] = g_sim.parameters.followedParticles[k];
}

}  /* extern "C" */
