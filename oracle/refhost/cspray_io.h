// cspray_io.h — TEST INFRASTRUCTURE ONLY.
//
// The part of class cspray (Multiphase/Multiphase/spray.h) that the
// reference's per-frame file writers and pouring emitters use, so that their
// text (spray.cu outputPovRaywater ... outputAirParticlePovRay, spray.cpp
// mapColorBlue2Red_h and CompPouringParam_*, taken unchanged by
// oracle/make_refhost.py) compiles for the host: the members they read, with
// the reference's names and types, and cudaMalloc / cudaMemcpy on host
// memory.  io.inc exports them to the tests.
#pragma once
#include "shim.h"
#include "utility.h"
#include <zlib.h>

#include <driver_types.h>   // cudaMemcpyKind
static inline int rh_memcpy(void* dst, const void* src, size_t n, cudaMemcpyKind) { memcpy(dst, src, n); return 0; }
#define cudaMemcpy rh_memcpy
static inline int rh_malloc(void** p, size_t n) { *p = malloc(n); return 0; }
#define cudaMalloc rh_malloc

bool verifyfloat3(float3& a);

class cspray {
public:
    char outputdir[30];                                    // spray.h:63
    bool mpause = false;
    uint maxVerts = 6000000, MCedgeNum = 1u << 26;         // spray.h:127, initMC (spray.cu:719-733)
    int parNumMax = 1 << 24;                               // spray.h:170
    float temperatureMax_render = 373, temperatureMin_render = 273;   // spray.h:296
    // the pouring emitters (spray.h:94, 138-141, spray.cpp:1416-1545)
    FlipConstant hparam;
    float pourRadius = 0;
    float3 pourpos, pourpos2, pourvel;
    float3 *dpourpos = nullptr, *dpourvel = nullptr;
    int pourNum = 0;
    void CompPouringParam_Freezing();
    void CompPouringParam_Ineraction();
    void CompPouringParam_Ineraction2();
    float3 mapColorBlue2Red_h(float v);
    void outputPovRaywater(int frame, float3* dpos, float3* dnormal, int pnum, uint* dindices, int indicesnum,
                           const char* objectname);
    void outputOBJwater(int frame, float3* dpos, float3* dnormal, int pnum, uint* dindices, int indicesnum,
                        const char* objectname);
    void outputBOBJwater(int frame, float3* dpos, float3* dnormal, int pnum, uint* dindices, int indicesnum,
                         const char* objectname);
    void outputColoredParticle(int frame, float3* dpos, float* dtemperature, int pnum);
    void outputSoloBubblePovRay(int frame, float3* dpos, float* dmass, char* dflag, int pnum);
    void outputAirParticlePovRay(int frame, float3* dpos, float* dmass, char* dflag, int pnum);
};
