// export.cpp — the reference's per-frame file writers, on host arrays.
//
// Reference (Multiphase/Multiphase/spray.cu): outputPovRaywater (2250-2306,
// POV-Ray mesh2), outputOBJwater (2308-2371, Wavefront OBJ), outputBOBJwater
// (2373-2438, gzip'd binary OBJ as read by Blender's fluid importer),
// outputColoredParticle (2440-2466), outputSoloBubblePovRay (2468-2496) and
// outputAirParticlePovRay (2498-2526) (POV-Ray spheres), with verifyfloat3
// (spray.cu:999-1008) and mapColorBlue2Red_h (spray.cpp:1299-1360). The text is
// produced with the reference's own printf formats, so files are byte-equal
// for equal inputs; the gzip stream is written by zlib at level 1 ("wb1"),
// as the reference does, so the uncompressed payload is byte-equal.
// Behaviours kept as the reference has them:
//   * an empty mesh gives an empty file (no header);
//   * a vertex or normal with a NaN component is written as (0, 0, 0);
//   * the BOBJ face block is preceded by the number of INDICES (3 per
//     triangle), not of triangles;
//   * OBJ indices are 1-based, POV-Ray and BOBJ indices 0-based.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <zlib.h>

#include "../../../include/mp.h"

namespace {

// verifyfloat3: false when a component is NaN (x > 0 || x < 1 holds for
// every other float, infinities included)
bool verify3(const float* v) {
    for (int a = 0; a < 3; a++)
        if (!(v[a] > 0 || v[a] < 1)) return false;
    return true;
}
void checked3(const float* src, float* dst) {
    if (verify3(src)) { dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2]; }
    else { dst[0] = dst[1] = dst[2] = 0.0f; }
}

struct File {
    FILE* f = nullptr;
    explicit File(const char* path) : f(std::fopen(path, "w")) {}
    ~File() { if (f) std::fclose(f); }
    // MP_OK when every write and the final flush succeeded
    int close() {
        bool ok = !std::ferror(f);
        ok = (std::fclose(f) == 0) && ok;
        f = nullptr;
        return ok ? MP_OK : MP_ERR_IO;
    }
};

int write_pov_mesh(const char* path, const char* name, const float* v, const float* nrm, int nv,
                   const uint32_t* idx, int ni) {
    File F(path);
    if (!F.f) return MP_ERR_IO;
    if (nv == 0) return F.close();
    FILE* fp = F.f;
    float q[3];
    std::fprintf(fp, "#declare watermesh=mesh2{\n");
    std::fprintf(fp, "vertex_vectors{\n");
    std::fprintf(fp, "%d,\n", nv);
    for (int i = 0; i < nv; i++) {
        checked3(v + 3 * (size_t)i, q);
        std::fprintf(fp, "< %f, %f, %f >,\n", q[0], q[1], q[2]);
    }
    std::fprintf(fp, "}\n ");
    std::fprintf(fp, "normal_vectors{\n");
    std::fprintf(fp, "%d,\n", nv);
    for (int i = 0; i < nv; i++) {
        checked3(nrm + 3 * (size_t)i, q);
        std::fprintf(fp, "<%f, %f, %f>,\n", q[0], q[1], q[2]);
    }
    std::fprintf(fp, "}\n ");
    std::fprintf(fp, "face_indices{\n");
    std::fprintf(fp, "%d,\n", ni / 3);
    for (int i = 0; i < ni; i += 3) std::fprintf(fp, "<%u, %u, %u>,\n", idx[i], idx[i + 1], idx[i + 2]);
    std::fprintf(fp, "}\n ");
    std::fprintf(fp, "inside_vector <0,0,1> }\n ");
    std::fprintf(fp, "object{ watermesh material{%s_material} }\n ", name);
    return F.close();
}

int write_obj_mesh(const char* path, const float* v, const float* nrm, int nv, const uint32_t* idx, int ni) {
    File F(path);
    if (!F.f) return MP_ERR_IO;
    if (nv == 0) return F.close();
    FILE* fp = F.f;
    float q[3];
    std::fprintf(fp, "#obj model\n");
    std::fprintf(fp, "#vertex_vectors\n");
    for (int i = 0; i < nv; i++) {
        checked3(v + 3 * (size_t)i, q);
        std::fprintf(fp, "v  %f %f %f\n", q[0], q[1], q[2]);
    }
    std::fprintf(fp, "#normal_vectors\n");
    for (int i = 0; i < nv; i++) {
        checked3(nrm + 3 * (size_t)i, q);
        std::fprintf(fp, "vn  %f %f %f\n", q[0], q[1], q[2]);
    }
    std::fprintf(fp, "#face_indices\n");
    for (int i = 0; i < ni; i += 3)
        std::fprintf(fp, "f  %d %d %d\n", (int)(idx[i] + 1), (int)(idx[i + 1] + 1), (int)(idx[i + 2] + 1));
    return F.close();
}

// the payload is assembled in memory and handed to zlib in one write; the
// reference's many small gzwrite calls give the same uncompressed stream
int write_bobj(const char* path, const float* v, const float* nrm, int nv, const uint32_t* idx, int ni) {
    gzFile gz = gzopen(path, "wb1");
    if (!gz) return MP_ERR_IO;
    if (nv == 0) return gzclose(gz) == Z_OK ? MP_OK : MP_ERR_IO;
    std::vector<unsigned char> buf;
    buf.reserve(4 + 12 * (size_t)nv + 4 + 12 * (size_t)nv + 4 + 4 * (size_t)ni);
    auto put = [&](const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        buf.insert(buf.end(), b, b + n);
    };
    float q[3];
    int32_t cnt = nv;
    put(&cnt, 4);
    for (int i = 0; i < nv; i++) { checked3(v + 3 * (size_t)i, q); put(q, 12); }
    put(&cnt, 4);
    for (int i = 0; i < nv; i++) { checked3(nrm + 3 * (size_t)i, q); put(q, 12); }
    int32_t nind = ni;
    put(&nind, 4);
    for (int i = 0; i < ni; i++) { int32_t t = (int32_t)idx[i]; put(&t, 4); }
    bool ok = true;
    size_t off = 0;
    while (ok && off < buf.size()) {
        unsigned chunk = (unsigned)std::min<size_t>(buf.size() - off, (size_t)1 << 30);
        ok = gzwrite(gz, buf.data() + off, chunk) == (int)chunk;
        off += chunk;
    }
    ok = (gzclose(gz) == Z_OK) && ok;
    return ok ? MP_OK : MP_ERR_IO;
}

// mapColorBlue2Red_h: v in [0, 6) walks blue -> cyan -> green -> yellow -> red
void blue2red(float v, float* c) {
    if (v < 0) { c[0] = 0.0f; c[1] = 0.0f; c[2] = 1.0f; return; }
    int ic = (int)v;
    float f = v - ic;
    switch (ic) {
    case 0: c[0] = 0; c[1] = f / 2; c[2] = 1; break;
    case 1: c[0] = 0; c[1] = f / 2 + 0.5f; c[2] = 1; break;
    case 2: c[0] = f / 2; c[1] = 1; c[2] = 1 - f / 2; break;
    case 3: c[0] = f / 2 + 0.5f; c[1] = 1; c[2] = 0.5f - f / 2; break;
    case 4: c[0] = 1; c[1] = 1.0f - f / 2; c[2] = 0; break;
    case 5: c[0] = 1; c[1] = 0.5f - f / 2; c[2] = 0; break;
    default: c[0] = 1; c[1] = 0; c[2] = 0; break;
    }
}

int write_particles(int kind, const char* path, const float* pos, const int8_t* flag, const float* T, int n,
                    float tmin, float tmax) {
    File F(path);
    if (!F.f) return MP_ERR_IO;
    FILE* fp = F.f;
    if (kind == MP_OUT_PARTICLES_COLORED) {
        const float iradius = 0.004f;
        float col[3];
        for (int i = 0; i < n; i++) {
            blue2red((T[i] - tmin) / (tmax - tmin) * 6.0f, col);
            std::fprintf(fp, "sphere{ <%f,%f,%f> %f texture{ finish{dropletFinish} pigment{ rgb<%f,%f,%f>}} }\n",
                         pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], iradius, col[0], col[1],
                         col[2]);
        }
    } else {
        const int want = kind == MP_OUT_PARTICLES_SOLO ? MP_TYPEAIRSOLO : MP_TYPEAIR;
        const float iradius = 0.005f;
        for (int i = 0; i < n; i++)
            if (flag[i] == want)
                std::fprintf(fp, "sphere{ <%f,%f,%f> %f texture{bblTexture} }\n", pos[3 * (size_t)i],
                             pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], iradius);
    }
    return F.close();
}

}  // namespace

extern "C" int mp_write_mesh(int format, const char* path, const char* object_name, const float* verts,
                             const float* normals, int nverts, const uint32_t* indices, int nindices) {
    if (!path || nverts < 0 || nindices < 0 || nindices % 3 != 0) return MP_ERR_ARG;
    if (nverts > 0 && (!verts || !normals)) return MP_ERR_ARG;
    if (nindices > 0 && !indices) return MP_ERR_ARG;
    for (int i = 0; i < nindices; i++)
        if (indices[i] >= (uint32_t)nverts) return MP_ERR_ARG;
    switch (format) {
    case MP_OUT_POV_MESH: return write_pov_mesh(path, object_name ? object_name : "", verts, normals, nverts, indices, nindices);
    case MP_OUT_OBJ_MESH: return write_obj_mesh(path, verts, normals, nverts, indices, nindices);
    case MP_OUT_BOBJ_GZ: return write_bobj(path, verts, normals, nverts, indices, nindices);
    default: return MP_ERR_ARG;
    }
}

extern "C" int mp_write_particles(int kind, const char* path, const float* pos, const int8_t* flag,
                                  const float* temperature, int n, float t_min, float t_max) {
    if (!path || n < 0) return MP_ERR_ARG;
    if (kind != MP_OUT_PARTICLES_COLORED && kind != MP_OUT_PARTICLES_SOLO && kind != MP_OUT_PARTICLES_AIR)
        return MP_ERR_ARG;
    if (n > 0 && !pos) return MP_ERR_ARG;
    if (n > 0 && kind == MP_OUT_PARTICLES_COLORED && !temperature) return MP_ERR_ARG;
    if (n > 0 && kind != MP_OUT_PARTICLES_COLORED && !flag) return MP_ERR_ARG;
    return write_particles(kind, path, pos, flag, temperature, n, t_min, t_max);
}
