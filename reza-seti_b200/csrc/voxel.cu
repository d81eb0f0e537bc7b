// GPU geometry pipeline: STL triangles -> the engine's node set.
//
// Replaces the reference's setup chain with the same results:
//   Reader::readSTLASCII            (GeometryReader.cpp:74-158)  -> lbm_stl_read_ascii
//   Geometry::GetBoundingbox ... excludeInletOutlet (ComplexGeometry.cpp:83-662)
//   SubDomain::CreateNodes / IdentifyNextToWallLattices / calculateBoundaryNormals
//                                    (Subdomain.cpp:364-572)      -> lbm_voxelise
// The reference labels every box point by the parity of a +z ray's hits
// against every triangle, with an MPI reduction per point (O(points x
// triangles)); here each vertical column of points first gets the list of
// triangles whose xy bounding box contains the column's ray, and one thread
// per point tests only those. The arithmetic of the hit test, the box-face
// ray offsets, the boundary / plane rules and the area / distance^2 weighted
// normals are the reference's, operation by operation; this file is built
// without FMA contraction (-fmad=false), so every double result rounds as the
// reference's g++ build (no FMA) rounds it and the node set is identical.
//
// Grid: spacing = 2 x grid_size (Geometry::DistributeTriangles doubles it),
// (nx + 1)(ny + 1)(nz + 1) points at bbox_min + i * spacing with
// nx = ceil((max_x - min_x) / spacing). Nodes are the fluid points in
// x-major, z-fastest order (SubDomain::GetFluidHaloLat, the order of
// Involved_Lat_), with coordinates = grid indices.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "errors.h"
#include "lbm_b200.h"
#include "lattice.cuh"

namespace {

using lbm::Lat;

// A triangle as the reference stores it (Struct.h Triangle): vertices, then
// the facet normal read from the file.
struct Tri {
    double x1, y1, z1, x2, y2, z2, x3, y3, z3, nx, ny, nz;
};

struct Grid {
    double min_x, max_x, min_y, max_y, min_z, max_z;
    double spacing;
    int nx, ny, nz;  // points per axis are n + 1
};

__host__ __device__ inline long long pidx(const Grid& g, int i, int j, int k) {
    return ((long long)i * (g.ny + 1) + j) * (g.nz + 1) + k;
}

// Geometry::isPointInsideTriangle (ComplexGeometry.cpp:208-262), with ray
// direction +z.
__device__ bool inside_triangle(double x, double y, double z, const Tri& t) {
    const double x1 = t.x1, y1 = t.y1, z1 = t.z1;
    const double x2 = t.x2, y2 = t.y2, z2 = t.z2;
    const double x3 = t.x3, y3 = t.y3, z3 = t.z3;
    const double dirX = 0.0, dirY = 0.0, dirZ = 1.0;
    const double uX = x2 - x1, uY = y2 - y1, uZ = z2 - z1;
    const double vX = x3 - x1, vY = y3 - y1, vZ = z3 - z1;
    const double nX = uY * vZ - uZ * vY;
    const double nY = uZ * vX - uX * vZ;
    const double nZ = uX * vY - uY * vX;
    const double nLengthSq = nX * nX + nY * nY + nZ * nZ;
    const double tol = 1e-16;
    if (nLengthSq < tol * tol) return false;
    const double w0X = x - x1, w0Y = y - y1, w0Z = z - z1;
    const double a = -(nX * w0X + nY * w0Y + nZ * w0Z);
    const double b = nX * dirX + nY * dirY + nZ * dirZ;
    if (fabs(b) < tol) return false;
    const double pos = a / b;
    const double ix = x + pos * dirX;
    const double iy = y + pos * dirY;
    const double iz = z + pos * dirZ;
    const double uu = uX * uX + uY * uY + uZ * uZ;
    const double uv = uX * vX + uY * vY + uZ * vZ;
    const double vv = vX * vX + vY * vY + vZ * vZ;
    const double wX = ix - x1, wY = iy - y1, wZ = iz - z1;
    const double wu = wX * uX + wY * uY + wZ * uZ;
    const double wv = wX * vX + wY * vY + wZ * vZ;
    const double D = uv * uv - uu * vv;
    const double s = (uv * wv - vv * wu) / D;
    if (s < 0.0 || s > 1.0) return false;
    const double tt = (uv * wu - uu * wv) / D;
    if (tt < 0.0 || (s + tt) > 1.0) return false;
    return true;
}

// The +z ray of point (i, j, k) after Geometry::adjustLineCoordinates, case 0
// (ComplexGeometry.cpp:313-345), and the ray end of labelPoints (:447-452).
struct Ray {
    double sx, sy, sz, ex, ey, ez;
};

__host__ __device__ inline Ray make_ray(const Grid& g, int i, int j, int k) {
    const double x = g.min_x + i * g.spacing;
    const double y = g.min_y + j * g.spacing;
    const double z = g.min_z + k * g.spacing;
    const double rayLength = g.max_z - g.min_z;
    Ray r{x, y, z, x, y, z + rayLength + 0.1};
    const double off = 0.01;
    if (r.sx == g.min_x) {
        r.sx += off;
        r.ex += off;
    }
    if (r.sx == g.max_x) {
        r.sx -= off;
        r.ex -= off;
    }
    if (r.sy == g.min_y) {
        r.sy += off;
        r.ey += off;
    }
    if (r.sy == g.max_y) {
        r.sy -= off;
        r.ey -= off;
    }
    if (r.sz == g.min_z) r.sz += off;
    if (r.ez == g.max_z) r.ez -= off;
    return r;
}

// Ray x, y of column (i, j): the z adjustments do not move them.
__host__ __device__ inline void column_xy(const Grid& g, int i, int j, double& x, double& y) {
    const Ray r = make_ray(g, i, j, 1);
    x = r.sx;
    y = r.sy;
}

// One triangle's column range: columns whose ray lies within its xy box
// (with a margin far above rounding); the inside test rejects the rest.
__device__ inline bool column_range(const Grid& g, const Tri& t, int& i0, int& i1, int& j0, int& j1, double& lx,
                                    double& hx, double& ly, double& hy) {
    lx = fmin(t.x1, fmin(t.x2, t.x3));
    hx = fmax(t.x1, fmax(t.x2, t.x3));
    ly = fmin(t.y1, fmin(t.y2, t.y3));
    hy = fmax(t.y1, fmax(t.y2, t.y3));
    const double mx = 1e-9 * (1.0 + fabs(lx) + fabs(hx)), my = 1e-9 * (1.0 + fabs(ly) + fabs(hy));
    lx -= mx;
    hx += mx;
    ly -= my;
    hy += my;
    // rays sit on the grid or 0.01 inside the box faces
    i0 = max(0, (int)floor((lx - g.min_x) / g.spacing) - 1);
    i1 = min(g.nx, (int)ceil((hx - g.min_x) / g.spacing) + 1);
    j0 = max(0, (int)floor((ly - g.min_y) / g.spacing) - 1);
    j1 = min(g.ny, (int)ceil((hy - g.min_y) / g.spacing) + 1);
    return i0 <= i1 && j0 <= j1;
}

__global__ void count_candidates(Grid g, const Tri* __restrict__ tris, long long n_tri, int* __restrict__ count) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tri) return;
    const Tri tr = tris[t];
    int i0, i1, j0, j1;
    double lx, hx, ly, hy;
    if (!column_range(g, tr, i0, i1, j0, j1, lx, hx, ly, hy)) return;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) {
            double x, y;
            column_xy(g, i, j, x, y);
            if (x >= lx && x <= hx && y >= ly && y <= hy) atomicAdd(count + (long long)i * (g.ny + 1) + j, 1);
        }
}

__global__ void fill_candidates(Grid g, const Tri* __restrict__ tris, long long n_tri, int* __restrict__ cursor,
                                int* __restrict__ cand) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tri) return;
    const Tri tr = tris[t];
    int i0, i1, j0, j1;
    double lx, hx, ly, hy;
    if (!column_range(g, tr, i0, i1, j0, j1, lx, hx, ly, hy)) return;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) {
            double x, y;
            column_xy(g, i, j, x, y);
            if (x >= lx && x <= hx && y >= ly && y <= hy)
                cand[atomicAdd(cursor + (long long)i * (g.ny + 1) + j, 1)] = (int)t;
        }
}

// Geometry::labelPoints (ComplexGeometry.cpp:435-514) with
// countIntersectinsTriangle (:265-310) over the column's candidates.
__global__ void label_points(Grid g, const Tri* __restrict__ tris, const long long* __restrict__ col_start,
                             const int* __restrict__ cand, unsigned char* __restrict__ fluid) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    if (p >= total) return;
    const int k = (int)(p % (g.nz + 1));
    const long long c = p / (g.nz + 1);
    const int j = (int)(c % (g.ny + 1));
    const int i = (int)(c / (g.ny + 1));
    const Ray r = make_ray(g, i, j, k);
    const double threshold = 1e-16;
    int count = 0;
    for (long long q = col_start[c]; q < col_start[c + 1]; ++q) {
        const Tri t = tris[cand[q]];
        const double px = r.sx, py = r.sy, pz = r.sz;
        const double dx = r.ex - r.sx, dy = r.ey - r.sy, dz = r.ez - r.sz;
        const double numerator = (t.x1 - px) * t.nx + (t.y1 - py) * t.ny + (t.z1 - pz) * t.nz;
        const double denominator = dx * t.nx + dy * t.ny + dz * t.nz;
        if (fabs(denominator) < threshold) continue;
        const double tt = numerator / denominator;
        if (tt >= 0.0 && tt <= 1.0) {
            const double ix = px + tt * dx, iy = py + tt * dy, iz = pz + tt * dz;
            if (inside_triangle(ix, iy, iz, t)) ++count;
        }
    }
    fluid[p] = (unsigned char)(count % 2 == 1);
}

struct Opening {
    int outlet, axis, index;  // index: outlet number (inlets: 0)
    double coord;
    double lo[3], hi[3];
};

// Point kinds: 0 not fluid, 1 fluid, 2 inlet, 3 outlet (outlet number in
// `which`), 4 wall — findBoundaryPoints (:517-564), getInOutBP (:567-641),
// excludeInletOutlet (:645-662), with CreateNodes' priority inlet > outlets
// in order > wall (Subdomain.cpp:392-428).
__global__ void classify_points(Grid g, const unsigned char* __restrict__ fluid, const Opening* __restrict__ ops,
                                int n_ops, unsigned char* __restrict__ kind, unsigned char* __restrict__ which) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    if (p >= total) return;
    if (!fluid[p]) {
        kind[p] = 0;
        return;
    }
    const int k = (int)(p % (g.nz + 1));
    const long long c = p / (g.nz + 1);
    const int j = (int)(c % (g.ny + 1));
    const int i = (int)(c / (g.ny + 1));
    bool bnd = false;
    for (int dx = -1; dx <= 1 && !bnd; ++dx)
        for (int dy = -1; dy <= 1 && !bnd; ++dy)
            for (int dz = -1; dz <= 1 && !bnd; ++dz) {
                const int a = i + dx, b = j + dy, e = k + dz;
                if (a >= 0 && a <= g.nx && b >= 0 && b <= g.ny && e >= 0 && e <= g.nz && !fluid[pidx(g, a, b, e)])
                    bnd = true;
            }
    if (i == 0 || i == g.nx || j == 0 || j == g.ny || k == 0 || k == g.nz) bnd = true;
    if (!bnd) {
        kind[p] = 1;
        return;
    }
    const double pt[3] = {g.min_x + i * g.spacing, g.min_y + j * g.spacing, g.min_z + k * g.spacing};
    int inlet = 0, outlet = -1;
    for (int o = 0; o < n_ops; ++o) {
        const Opening& op = ops[o];
        bool hit = fabs(pt[op.axis] - op.coord) <= 2.5e-2;
        for (int a = 0; a < 3 && hit; ++a)
            if (a != op.axis) hit = pt[a] >= op.lo[a] && pt[a] <= op.hi[a];
        if (!hit) continue;
        if (!op.outlet) inlet = 1;
        else if (outlet < 0) outlet = op.index;
    }
    if (inlet) {
        kind[p] = 2;
    } else if (outlet >= 0) {
        kind[p] = 3;
        which[p] = (unsigned char)outlet;
    } else {
        kind[p] = 4;
    }
}

__global__ void column_counts(Grid g, const unsigned char* __restrict__ kind, int* __restrict__ count) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)(g.nx + 1) * (g.ny + 1)) return;
    int n = 0;
    for (int k = 0; k <= g.nz; ++k) n += kind[c * (g.nz + 1) + k] != 0;
    count[c] = n;
}

__global__ void compact_nodes(Grid g, const unsigned char* __restrict__ kind, const long long* __restrict__ start,
                              int* __restrict__ node_of, int* __restrict__ coords, unsigned char* __restrict__ nkind) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)(g.nx + 1) * (g.ny + 1)) return;
    const int j = (int)(c % (g.ny + 1)), i = (int)(c / (g.ny + 1));
    long long n = start[c];
    for (int k = 0; k <= g.nz; ++k) {
        const long long p = c * (g.nz + 1) + k;
        if (!kind[p]) {
            node_of[p] = -1;
            continue;
        }
        node_of[p] = (int)n;
        coords[3 * n] = i;
        coords[3 * n + 1] = j;
        coords[3 * n + 2] = k;
        nkind[n] = kind[p];
        ++n;
    }
}

// SubDomain::IdentifyNextToWallLattices (Subdomain.cpp:475-493): plain fluid
// D3Q19 neighbours of wall nodes.
__global__ void mark_nearwall(Grid g, long long n, const int* __restrict__ coords, const unsigned char* __restrict__ nkind,
                              const int* __restrict__ node_of, unsigned char* __restrict__ near) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || nkind[v] != 4) return;
    using L = Lat<19>;
    for (int q = 0; q < 19; ++q) {
        const int a = coords[3 * v] + L::cx(q), b = coords[3 * v + 1] + L::cy(q), e = coords[3 * v + 2] + L::cz(q);
        if (a < 0 || a > g.nx || b < 0 || b > g.ny || e < 0 || e > g.nz) continue;
        const int m = node_of[pidx(g, a, b, e)];
        if (m >= 0 && nkind[m] == 1) near[m] = 1;
    }
}

// SubDomain::calculateBoundaryNormals (Subdomain.cpp:499-572): facet normals
// from the vertices, weighted by area / distance^2 to the facet centroid,
// summed over all triangles in file order.
__global__ void nearwall_normals(Grid g, const Tri* __restrict__ tris, long long n_tri, int n_nw,
                                 const int* __restrict__ nw_coords, double* __restrict__ out) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_nw) return;
    const double x = g.min_x + nw_coords[3 * w] * g.spacing;
    const double y = g.min_y + nw_coords[3 * w + 1] * g.spacing;
    const double z = g.min_z + nw_coords[3 * w + 2] * g.spacing;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (long long t = 0; t < n_tri; ++t) {
        const Tri tr = tris[t];
        const double ux = tr.x2 - tr.x1, uy = tr.y2 - tr.y1, uz = tr.z2 - tr.z1;
        const double vx = tr.x3 - tr.x1, vy = tr.y3 - tr.y1, vz = tr.z3 - tr.z1;
        double nx = uy * vz - uz * vy;
        double ny = uz * vx - ux * vz;
        double nz = ux * vy - uy * vx;
        const double norm = sqrt(nx * nx + ny * ny + nz * nz);
        if (norm > 0) {
            nx /= norm;
            ny /= norm;
            nz /= norm;
        }
        const double area = 0.5 * norm;
        const double cx = (tr.x1 + tr.x2 + tr.x3) / 3.0;
        const double cy = (tr.y1 + tr.y2 + tr.y3) / 3.0;
        const double cz = (tr.z1 + tr.z2 + tr.z3) / 3.0;
        // std::pow(d, 2) is exactly d * d (one rounding either way)
        const double dxx = x - cx, dyy = y - cy, dzz = z - cz;
        const double distance = sqrt(dxx * dxx + dyy * dyy + dzz * dzz);
        const double weight = area / (distance * distance);
        s0 += nx * weight;
        s1 += ny * weight;
        s2 += nz * weight;
    }
    const double norm = sqrt(s0 * s0 + s1 * s1 + s2 * s2);
    if (norm > 0) {
        s0 /= norm;
        s1 /= norm;
        s2 /= norm;
    }
    out[3 * (long long)w] = s0;
    out[3 * (long long)w + 1] = s1;
    out[3 * (long long)w + 2] = s2;
}

struct DevBufs {
    std::vector<void*> p;
    cudaError_t err = cudaSuccess;
    template <class T>
    T* get(size_t n) {
        if (err != cudaSuccess) return nullptr;
        void* q = nullptr;
        err = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (err != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T*)q;
    }
    ~DevBufs() {
        for (void* q : p) cudaFree(q);
    }
};

unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Host result: the node set and lists in lbm_desc form.
struct lbm_voxel {
    Grid g{};
    std::vector<int32_t> coords;
    std::vector<uint8_t> kind;  // lbm_node_kind
    std::vector<int64_t> inlet, wall, nearwall;
    std::vector<int64_t> outlet_offsets, outlet_nodes;
    std::vector<double> outlet_normals, nearwall_normals;
    double inlet_normal[3] = {0, 0, 0};
    int n_outlets = 0;
    double ms = 0.0;
};

extern "C" {

int lbm_stl_read_ascii(const char* path, int64_t* n_triangles, double** triangles) {
    if (!path || !n_triangles || !triangles) return LBM_ERR_ARGUMENT;
    std::ifstream file(path);
    if (!file.is_open()) {
        lbm::set_global_error(std::string("cannot open ") + path);
        return LBM_ERR_ARGUMENT;
    }
    // the line grammar of Reader::readSTLASCII: "facet normal nx ny nz",
    // "outer loop", three "vertex x y z", "endloop", "endfacet". The
    // reference skips a facet whose lines do not follow it (and keeps the
    // previous facet's vertices where a vertex line fails), without a word;
    // here a facet that does not follow it, or a file that ends inside one,
    // is an error naming the line, and so is a file without facets.
    std::vector<double> out;
    std::string line, w1, w2;
    long long lineno = 0;
    auto bad = [&](const char* what) {
        lbm::set_global_error(std::string(path) + ":" + std::to_string(lineno) + ": " + what);
        return LBM_ERR_ARGUMENT;
    };
    auto next = [&](std::stringstream& ss) {
        if (!std::getline(file, line)) return false;
        ++lineno;
        ss.clear();
        ss.str(line);
        return true;
    };
    std::stringstream ss;
    while (next(ss)) {
        double n[3];
        if (!(ss >> w1) || w1 != "facet") continue;  // solid / endsolid / blank lines
        if (!(ss >> w2 >> n[0] >> n[1] >> n[2]) || w2 != "normal") return bad("malformed facet normal line");
        if (!next(ss)) return bad("file ends inside a facet");
        if (!(ss >> w1 >> w2) || w1 != "outer" || w2 != "loop") return bad("expected outer loop");
        double v[9];
        for (int i = 0; i < 3; ++i) {
            if (!next(ss)) return bad("file ends inside a facet");
            if (!(ss >> w1 >> v[3 * i] >> v[3 * i + 1] >> v[3 * i + 2]) || w1 != "vertex")
                return bad("malformed vertex line");
        }
        if (!next(ss)) return bad("file ends inside a facet");
        if (!(ss >> w1) || w1 != "endloop") return bad("expected endloop");
        if (!next(ss)) return bad("file ends inside a facet");
        if (!(ss >> w1) || w1 != "endfacet") return bad("expected endfacet");
        for (int i = 0; i < 9; ++i) out.push_back(v[i]);
        for (int i = 0; i < 3; ++i) out.push_back(n[i]);
    }
    if (out.empty()) {
        lbm::set_global_error(std::string(path) + ": no facets");
        return LBM_ERR_ARGUMENT;
    }
    double* buf = (double*)std::malloc(out.size() * sizeof(double));
    if (!buf) return LBM_ERR_ARGUMENT;
    std::memcpy(buf, out.data(), out.size() * sizeof(double));
    *triangles = buf;
    *n_triangles = (int64_t)(out.size() / 12);
    return LBM_OK;
}

void lbm_free(void* p) { std::free(p); }

int lbm_voxelise(const lbm_voxel_desc* d, lbm_voxel** out) {
    using Clock = std::chrono::steady_clock;
    if (!d || !out) return LBM_ERR_ARGUMENT;
    *out = nullptr;
    auto fail = [](int code, const std::string& m) {
        lbm::set_global_error(m);
        return code;
    };
    if (d->n_triangles <= 0 || !d->triangles) return fail(LBM_ERR_ARGUMENT, "no triangles");
    if (!(d->grid_size > 0)) return fail(LBM_ERR_ARGUMENT, "grid_size must be positive");
    if (d->n_openings < 0 || (d->n_openings > 0 && !d->openings)) return fail(LBM_ERR_ARGUMENT, "bad openings");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
    if (d->device < 0 || d->device >= ndev) return fail(LBM_ERR_ARGUMENT, "device ordinal out of range");
    cudaSetDevice(d->device);
    const auto t_start = Clock::now();

    const int64_t nt = d->n_triangles;
    std::vector<Tri> tris(nt);
    std::memcpy(tris.data(), d->triangles, sizeof(Tri) * nt);
    Grid g{};
    g.min_x = g.min_y = g.min_z = INFINITY;
    g.max_x = g.max_y = g.max_z = -INFINITY;
    for (const Tri& t : tris) {
        g.min_x = std::min(g.min_x, std::min(t.x1, std::min(t.x2, t.x3)));
        g.min_y = std::min(g.min_y, std::min(t.y1, std::min(t.y2, t.y3)));
        g.min_z = std::min(g.min_z, std::min(t.z1, std::min(t.z2, t.z3)));
        g.max_x = std::max(g.max_x, std::max(t.x1, std::max(t.x2, t.x3)));
        g.max_y = std::max(g.max_y, std::max(t.y1, std::max(t.y2, t.y3)));
        g.max_z = std::max(g.max_z, std::max(t.z1, std::max(t.z2, t.z3)));
    }
    g.spacing = d->grid_size;
    g.spacing *= 2;
    const double ex = std::ceil((g.max_x - g.min_x) / g.spacing), ey = std::ceil((g.max_y - g.min_y) / g.spacing),
                 ez = std::ceil((g.max_z - g.min_z) / g.spacing);
    if (!(ex < 65536 && ey < 65536 && ez < 65536) || (ex + 1) * (ey + 1) * (ez + 1) > 4.0e9)
        return fail(LBM_ERR_ARGUMENT, "grid too large for grid_size");
    g.nx = (int)ex;
    g.ny = (int)ey;
    g.nz = (int)ez;
    const long long ncol = (long long)(g.nx + 1) * (g.ny + 1);
    const long long npts = ncol * (g.nz + 1);

    std::vector<Opening> ops;
    int n_out = 0;
    const lbm_opening* last_inlet = nullptr;
    for (int o = 0; o < d->n_openings; ++o) {
        const lbm_opening& s = d->openings[o];
        if (s.axis < 0 || s.axis > 2) return fail(LBM_ERR_ARGUMENT, "opening axis must be 0, 1 or 2");
        Opening op{};
        op.outlet = s.outlet != 0;
        op.axis = s.axis;
        op.index = op.outlet ? n_out++ : 0;
        op.coord = s.coordinate;
        for (int a = 0; a < 3; ++a) {
            op.lo[a] = s.range[a][0];
            op.hi[a] = s.range[a][1];
        }
        if (!op.outlet) last_inlet = &s;
        ops.push_back(op);
    }
    if (n_out > 255) return fail(LBM_ERR_ARGUMENT, "too many outlets");
    // the reference only warns (ComplexGeometry.cpp:667-672) and then runs a
    // simulation that nothing drives
    if (!last_inlet) return fail(LBM_ERR_ARGUMENT, "no inlet opening given");

    DevBufs B;
    Tri* d_tris = B.get<Tri>(nt);
    int* d_count = B.get<int>(ncol);
    long long* d_start = B.get<long long>(ncol + 1);
    unsigned char* d_fluid = B.get<unsigned char>(npts);
    unsigned char* d_kind = B.get<unsigned char>(npts);
    unsigned char* d_which = B.get<unsigned char>(npts);
    Opening* d_ops = B.get<Opening>(std::max<size_t>(ops.size(), 1));
    if (B.err != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("voxeliser buffers: ") + cudaGetErrorString(B.err));
    cudaMemcpy(d_tris, tris.data(), sizeof(Tri) * nt, cudaMemcpyHostToDevice);
    if (!ops.empty()) cudaMemcpy(d_ops, ops.data(), sizeof(Opening) * ops.size(), cudaMemcpyHostToDevice);
    cudaMemset(d_count, 0, sizeof(int) * ncol);
    cudaMemset(d_which, 0, npts);
    const int T = 256;

    // candidate triangles per column (CSR)
    count_candidates<<<blocks(nt, T), T>>>(g, d_tris, nt, d_count);
    std::vector<int> cnt(ncol);
    cudaMemcpy(cnt.data(), d_count, sizeof(int) * ncol, cudaMemcpyDeviceToHost);
    std::vector<long long> start(ncol + 1, 0);
    for (long long c = 0; c < ncol; ++c) start[c + 1] = start[c] + cnt[c];
    int* d_cand = B.get<int>((size_t)start[ncol]);
    if (B.err != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("voxeliser candidates: ") + cudaGetErrorString(B.err));
    {
        std::vector<int> cur(start.begin(), start.end() - 1);
        for (long long c = 0; c < ncol; ++c)
            if (start[c] > INT32_MAX) return fail(LBM_ERR_ARGUMENT, "too many column candidates");
        cudaMemcpy(d_count, cur.data(), sizeof(int) * ncol, cudaMemcpyHostToDevice);
    }
    cudaMemcpy(d_start, start.data(), sizeof(long long) * (ncol + 1), cudaMemcpyHostToDevice);
    fill_candidates<<<blocks(nt, T), T>>>(g, d_tris, nt, d_count, d_cand);
    label_points<<<blocks(npts, T), T>>>(g, d_tris, d_start, d_cand, d_fluid);
    classify_points<<<blocks(npts, T), T>>>(g, d_fluid, d_ops, (int)ops.size(), d_kind, d_which);

    // compaction: nodes in x-major, z-fastest order
    column_counts<<<blocks(ncol, T), T>>>(g, d_kind, d_count);
    cudaMemcpy(cnt.data(), d_count, sizeof(int) * ncol, cudaMemcpyDeviceToHost);
    for (long long c = 0; c < ncol; ++c) start[c + 1] = start[c] + cnt[c];
    const long long n = start[ncol];
    if (n == 0) return fail(LBM_ERR_ARGUMENT, "the STL encloses no grid point");
    if (n > INT32_MAX - 256) return fail(LBM_ERR_ARGUMENT, "too many nodes");
    cudaMemcpy(d_start, start.data(), sizeof(long long) * (ncol + 1), cudaMemcpyHostToDevice);
    int* d_node_of = B.get<int>(npts);
    int* d_coords = B.get<int>(3 * n);
    unsigned char* d_nkind = B.get<unsigned char>(n);
    unsigned char* d_near = B.get<unsigned char>(n);
    if (B.err != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("voxeliser nodes: ") + cudaGetErrorString(B.err));
    cudaMemset(d_near, 0, n);
    compact_nodes<<<blocks(ncol, T), T>>>(g, d_kind, d_start, d_node_of, d_coords, d_nkind);
    mark_nearwall<<<blocks(n, T), T>>>(g, n, d_coords, d_nkind, d_node_of, d_near);

    auto* v = new lbm_voxel();
    v->g = g;
    v->coords.resize(3 * n);
    std::vector<unsigned char> nk(n), near(n);
    cudaMemcpy(v->coords.data(), d_coords, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(nk.data(), d_nkind, n, cudaMemcpyDeviceToHost);
    cudaMemcpy(near.data(), d_near, n, cudaMemcpyDeviceToHost);
    // outlet numbers of the outlet nodes
    std::vector<unsigned char> which_pts;
    std::vector<std::vector<int64_t>> outs(n_out);
    v->kind.resize(n);
    {
        std::vector<unsigned char> which(npts);
        cudaMemcpy(which.data(), d_which, npts, cudaMemcpyDeviceToHost);
        for (long long i = 0; i < n; ++i) {
            const int* c = &v->coords[3 * i];
            switch (nk[i]) {
                case 1: v->kind[i] = LBM_NODE_FLUID; break;
                case 2:
                    v->kind[i] = LBM_NODE_INLET;
                    v->inlet.push_back(i);
                    break;
                case 3:
                    v->kind[i] = LBM_NODE_OUTLET;
                    outs[which[pidx(g, c[0], c[1], c[2])]].push_back(i);
                    break;
                default:
                    v->kind[i] = LBM_NODE_WALL;
                    v->wall.push_back(i);
                    break;
            }
            if (near[i]) v->nearwall.push_back(i);
        }
    }
    if (v->inlet.empty()) {
        delete v;
        return fail(LBM_ERR_ARGUMENT, "the inlet opening matches no grid point (check its plane and coordinate "
                                      "against the STL's bounding box)");
    }
    v->n_outlets = n_out;
    v->outlet_offsets.push_back(0);
    for (int o = 0; o < n_out; ++o) {
        v->outlet_nodes.insert(v->outlet_nodes.end(), outs[o].begin(), outs[o].end());
        v->outlet_offsets.push_back((int64_t)v->outlet_nodes.size());
    }
    for (int o = 0; o < d->n_openings; ++o)
        if (d->openings[o].outlet)
            for (int a = 0; a < 3; ++a) v->outlet_normals.push_back(d->openings[o].normal[a]);
    if (last_inlet)
        for (int a = 0; a < 3; ++a) v->inlet_normal[a] = last_inlet->normal[a];

    // near-wall normals
    const int n_nw = (int)v->nearwall.size();
    v->nearwall_normals.assign(3 * (size_t)n_nw, 0.0);
    if (n_nw) {
        std::vector<int> nwc(3 * (size_t)n_nw);
        for (int w = 0; w < n_nw; ++w)
            for (int a = 0; a < 3; ++a) nwc[3 * (size_t)w + a] = v->coords[3 * v->nearwall[w] + a];
        int* d_nwc = B.get<int>(nwc.size());
        double* d_nrm = B.get<double>(nwc.size());
        if (B.err != cudaSuccess) {
            delete v;
            return fail(LBM_ERR_CUDA, std::string("voxeliser normals: ") + cudaGetErrorString(B.err));
        }
        cudaMemcpy(d_nwc, nwc.data(), sizeof(int) * nwc.size(), cudaMemcpyHostToDevice);
        nearwall_normals<<<blocks(n_nw, 128), 128>>>(g, d_tris, nt, n_nw, d_nwc, d_nrm);
        cudaMemcpy(v->nearwall_normals.data(), d_nrm, sizeof(double) * nwc.size(), cudaMemcpyDeviceToHost);
    }
    cudaError_t ce = cudaDeviceSynchronize();
    if (ce == cudaSuccess) ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        delete v;
        return fail(LBM_ERR_CUDA, std::string("voxeliser: ") + cudaGetErrorString(ce));
    }
    v->ms = std::chrono::duration<double, std::milli>(Clock::now() - t_start).count();
    *out = v;
    return LBM_OK;
}

int lbm_voxel_info(const lbm_voxel* v, int32_t dims[3], double origin[3], double* spacing, int64_t* n_nodes,
                   int64_t* n_nearwall, double* build_ms) {
    if (!v) return LBM_ERR_ARGUMENT;
    if (dims) {
        dims[0] = v->g.nx + 1;
        dims[1] = v->g.ny + 1;
        dims[2] = v->g.nz + 1;
    }
    if (origin) {
        origin[0] = v->g.min_x;
        origin[1] = v->g.min_y;
        origin[2] = v->g.min_z;
    }
    if (spacing) *spacing = v->g.spacing;
    if (n_nodes) *n_nodes = (int64_t)v->kind.size();
    if (n_nearwall) *n_nearwall = (int64_t)v->nearwall.size();
    if (build_ms) *build_ms = v->ms;
    return LBM_OK;
}

int lbm_voxel_describe(const lbm_voxel* v, lbm_desc* d) {
    if (!v || !d) return LBM_ERR_ARGUMENT;
    d->n_nodes = (int64_t)v->kind.size();
    d->coords = v->coords.data();
    d->kind = v->kind.data();
    d->n_inlet = (int64_t)v->inlet.size();
    d->inlet = v->inlet.data();
    for (int a = 0; a < 3; ++a) d->inlet_normal[a] = v->inlet_normal[a];
    d->n_outlets = v->n_outlets;
    d->outlet_offsets = v->outlet_offsets.data();
    d->outlet_nodes = v->outlet_nodes.data();
    d->outlet_normals = v->outlet_normals.data();
    d->n_wall = (int64_t)v->wall.size();
    d->wall = v->wall.data();
    d->n_nearwall = (int64_t)v->nearwall.size();
    d->nearwall = v->nearwall.data();
    d->nearwall_normals = v->nearwall_normals.data();
    d->spacing = v->g.spacing;
    return LBM_OK;
}

int lbm_voxel_destroy(lbm_voxel* v) {
    delete v;
    return LBM_OK;
}

}  // extern "C"
