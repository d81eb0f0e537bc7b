// Result files of the reference's output step (Simulation::WriteOutput,
// Simulation.cpp:835-856) without VTK:
//   * lbm_write_surface_csv  — OutputFile::WriteSurfaceAttribute
//     (OutputFile.cpp:234-316): one row per near-wall node, in the near-wall
//     list's order, "X,Y,Z,WSS[,OSI,TAWSS],VelMag", numbers in the ostream
//     default format (6 significant digits);
//   * lbm_smooth_surface_csv — OutputFile::processFlowData / smoothData
//     (:395-483): re-reads that file and replaces WSS (and OSI, TAWSS) by the
//     mean over the other rows within the search radius. The reference pairs
//     every row with every row (O(N^2)); here the rows are binned into cells
//     of the radius, and a GPU thread per row gathers the rows of its 27
//     neighbouring cells, keeps those within the radius, and sums them in
//     file order — the reference's neighbour set and summation order, so the
//     written numbers are the same;
//   * lbm_write_vtu          — OutputFile::WriteVTK_Collective (:60-230): the
//     nodes in its point order (z, then y, then x fastest), Velocity, Density
//     and VelocityMagnitude per point, and a hexahedron for every lattice cell
//     whose 8 corners are nodes. VTK's own encoder is not available, so the
//     file is VTK XML with raw appended binary data (readable by VTK and
//     ParaView), not VTK's byte stream; points are Float32, as vtkPoints
//     stores them by default.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "engine_view.h"
#include "errors.h"
#include "lbm_b200.h"

namespace {

struct Row {
    double x, y, z, wss, osi, tawss, vel;
};

constexpr int MAX_NEIGHBOURS = 128;

// Mean of the other rows within `radius` (OutputFile::calculateMeanNeighboringValues,
// :325-366), for WSS, OSI and TAWSS. Cells of size h >= radius: a row's
// neighbours lie in its own or an adjacent cell. A row with more than
// MAX_NEIGHBOURS candidates in range is flagged for the host.
__global__ void smooth_rows(int n, const Row* __restrict__ rows, const long long* __restrict__ keys,
                            const int* __restrict__ order, double radius, double h, double x0, double y0, double z0,
                            long long ny, long long nz, int pulsatile, double* __restrict__ out, int* __restrict__ overflow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Row p = rows[i];
    const long long cx = (long long)floor((p.x - x0) / h), cy = (long long)floor((p.y - y0) / h),
                    cz = (long long)floor((p.z - z0) / h);
    int found[MAX_NEIGHBOURS];
    int nf = 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                const long long key = ((cx + dx) * ny + (cy + dy)) * nz + (cz + dz);
                // first sorted entry with this key
                int lo = 0, hi = n;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (keys[mid] < key) lo = mid + 1;
                    else hi = mid;
                }
                for (int s = lo; s < n && keys[s] == key; ++s) {
                    const int j = order[s];
                    const Row q = rows[j];
                    // calculateDistance (:319-322): std::pow(d, 2) is d * d
                    const double ddx = q.x - p.x, ddy = q.y - p.y, ddz = q.z - p.z;
                    const double d = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                    if (d > 0 && d <= radius) {
                        if (nf == MAX_NEIGHBOURS) {
                            overflow[i] = 1;
                            return;
                        }
                        found[nf++] = j;
                    }
                }
            }
    // file order
    for (int a = 1; a < nf; ++a) {
        const int v = found[a];
        int b = a - 1;
        while (b >= 0 && found[b] > v) {
            found[b + 1] = found[b];
            --b;
        }
        found[b + 1] = v;
    }
    double sw = 0.0, so = 0.0, st = 0.0;
    for (int a = 0; a < nf; ++a) {
        sw += rows[found[a]].wss;
        so += rows[found[a]].osi;
        st += rows[found[a]].tawss;
    }
    out[3 * (long long)i] = nf > 0 ? sw / nf : p.wss;
    out[3 * (long long)i + 1] = pulsatile ? (nf > 0 ? so / nf : p.osi) : p.osi;
    out[3 * (long long)i + 2] = pulsatile ? (nf > 0 ? st / nf : p.tawss) : p.tawss;
}

int fail(int code, const std::string& m) {
    lbm::set_global_error(m);
    return code;
}

}  // namespace

extern "C" {

int lbm_write_surface_csv(lbm_engine* e, const char* path, const double origin[3], double spacing,
                          int32_t pulsatile) {
    lbm::EngineView v;
    if (!e || !path || !origin || !lbm::engine_view(e, v)) return LBM_ERR_ARGUMENT;
    std::vector<double> rho(v.n), u(3 * v.n), wss(v.n_nw), osi(v.n_nw), tawss(v.n_nw);
    if (int rc = lbm_get_macros(e, rho.data(), u.data())) return rc;
    if (int rc = lbm_get_wss(e, wss.data(), nullptr, nullptr)) return rc;
    if (pulsatile)
        if (int rc = lbm_get_osi_tawss(e, osi.data(), tawss.data())) return rc;
    std::ofstream f(path);
    if (!f) return fail(LBM_ERR_ARGUMENT, std::string("cannot write ") + path);
    f << "X,Y,Z,WSS";
    if (pulsatile) f << ",OSI,TAWSS";
    f << ",VelMag\n";
    for (int64_t k = 0; k < v.n_nw; ++k) {
        const int64_t n = v.nearwall[k];
        const double x = origin[0] + v.coords[3 * n] * spacing;
        const double y = origin[1] + v.coords[3 * n + 1] * spacing;
        const double z = origin[2] + v.coords[3 * n + 2] * spacing;
        const double* un = &u[3 * n];
        const double vel = std::sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
        f << x << "," << y << "," << z << "," << wss[k];
        if (pulsatile) f << "," << osi[k] << "," << tawss[k];
        f << "," << vel << "\n";
    }
    return f.good() ? LBM_OK : fail(LBM_ERR_ARGUMENT, std::string("error writing ") + path);
}

int lbm_smooth_surface_csv(const char* in_path, const char* out_path, double radius, int32_t pulsatile,
                           int32_t device) {
    if (!in_path || !out_path || !(radius > 0)) return LBM_ERR_ARGUMENT;
    std::ifstream in(in_path);
    if (!in) return fail(LBM_ERR_ARGUMENT, std::string("cannot open ") + in_path);
    std::string header, line;
    if (!std::getline(in, header)) return fail(LBM_ERR_ARGUMENT, "empty surface file");
    // row grammar of processFlowData: comma-separated std::stod fields; a
    // row that does not parse is dropped
    std::vector<Row> rows;
    while (std::getline(in, line)) {
        std::stringstream ss(line);
        std::string tok;
        Row r{};
        try {
            std::getline(ss, tok, ',');
            r.x = std::stod(tok);
            std::getline(ss, tok, ',');
            r.y = std::stod(tok);
            std::getline(ss, tok, ',');
            r.z = std::stod(tok);
            std::getline(ss, tok, ',');
            r.wss = std::stod(tok);
            if (pulsatile) {
                std::getline(ss, tok, ',');
                r.osi = std::stod(tok);
                std::getline(ss, tok, ',');
                r.tawss = std::stod(tok);
            }
            std::getline(ss, tok, ',');
            r.vel = std::stod(tok);
            rows.push_back(r);
        } catch (const std::exception&) {
        }
    }
    const int n = (int)rows.size();
    std::vector<double> sm(3 * (size_t)std::max(n, 1));
    if (n > 0) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device");
        if (device < 0 || device >= ndev) return fail(LBM_ERR_ARGUMENT, "device ordinal out of range");
        cudaSetDevice(device);
        // cells slightly larger than the radius; sorted cell keys
        const double h = radius * (1.0 + 1e-9);
        double x0 = INFINITY, y0 = INFINITY, z0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY, z1 = -INFINITY;
        for (const Row& r : rows) {
            x0 = std::min(x0, r.x), y0 = std::min(y0, r.y), z0 = std::min(z0, r.z);
            x1 = std::max(x1, r.x), y1 = std::max(y1, r.y), z1 = std::max(z1, r.z);
        }
        // one empty cell of margin on each side keeps neighbour keys in range
        x0 -= h, y0 -= h, z0 -= h;
        const long long ny = (long long)std::floor((y1 - y0) / h) + 3, nz = (long long)std::floor((z1 - z0) / h) + 3;
        const long long nxl = (long long)std::floor((x1 - x0) / h) + 3;
        if ((double)nxl * ny * nz > 9.0e18) return fail(LBM_ERR_ARGUMENT, "search radius too small for the extent");
        std::vector<long long> key(n);
        for (int i = 0; i < n; ++i)
            key[i] = ((long long)std::floor((rows[i].x - x0) / h) * ny + (long long)std::floor((rows[i].y - y0) / h)) *
                         nz + (long long)std::floor((rows[i].z - z0) / h);
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
        std::vector<long long> skey(n);
        for (int i = 0; i < n; ++i) skey[i] = key[order[i]];
        Row* d_rows = nullptr;
        long long* d_keys = nullptr;
        int *d_order = nullptr, *d_over = nullptr;
        double* d_out = nullptr;
        cudaError_t ce = cudaMalloc(&d_rows, sizeof(Row) * n);
        if (ce == cudaSuccess) ce = cudaMalloc(&d_keys, sizeof(long long) * n);
        if (ce == cudaSuccess) ce = cudaMalloc(&d_order, sizeof(int) * n);
        if (ce == cudaSuccess) ce = cudaMalloc(&d_over, sizeof(int) * n);
        if (ce == cudaSuccess) ce = cudaMalloc(&d_out, sizeof(double) * 3 * n);
        std::vector<int> over(n, 0);
        if (ce == cudaSuccess) {
            cudaMemcpy(d_rows, rows.data(), sizeof(Row) * n, cudaMemcpyHostToDevice);
            cudaMemcpy(d_keys, skey.data(), sizeof(long long) * n, cudaMemcpyHostToDevice);
            cudaMemcpy(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
            cudaMemset(d_over, 0, sizeof(int) * n);
            // keys were formed with x0 shifted; the kernel sees the same origin
            smooth_rows<<<(n + 127) / 128, 128>>>(n, d_rows, d_keys, d_order, radius, h, x0, y0, z0, ny, nz,
                                                  pulsatile, d_out, d_over);
            ce = cudaMemcpy(sm.data(), d_out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
            if (ce == cudaSuccess) ce = cudaMemcpy(over.data(), d_over, sizeof(int) * n, cudaMemcpyDeviceToHost);
        }
        cudaFree(d_rows);
        cudaFree(d_keys);
        cudaFree(d_order);
        cudaFree(d_over);
        cudaFree(d_out);
        if (ce != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("smoothing: ") + cudaGetErrorString(ce));
        // rows with very many neighbours: the reference's loop on the host
        for (int i = 0; i < n; ++i) {
            if (!over[i]) continue;
            double sw = 0, so = 0, st = 0;
            int c = 0;
            for (int j = 0; j < n; ++j) {
                const double dx = rows[j].x - rows[i].x, dy = rows[j].y - rows[i].y, dz = rows[j].z - rows[i].z;
                const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (d > 0 && d <= radius) {
                    sw += rows[j].wss;
                    so += rows[j].osi;
                    st += rows[j].tawss;
                    ++c;
                }
            }
            sm[3 * (size_t)i] = c ? sw / c : rows[i].wss;
            sm[3 * (size_t)i + 1] = pulsatile ? (c ? so / c : rows[i].osi) : rows[i].osi;
            sm[3 * (size_t)i + 2] = pulsatile ? (c ? st / c : rows[i].tawss) : rows[i].tawss;
        }
    }
    std::ofstream out(out_path);
    if (!out) return fail(LBM_ERR_ARGUMENT, std::string("cannot write ") + out_path);
    out << header << std::endl;
    for (int i = 0; i < n; ++i) {
        out << rows[i].x << "," << rows[i].y << "," << rows[i].z << "," << sm[3 * (size_t)i];
        if (pulsatile) out << "," << sm[3 * (size_t)i + 1] << "," << sm[3 * (size_t)i + 2];
        out << "," << rows[i].vel << std::endl;
    }
    return out.good() ? LBM_OK : fail(LBM_ERR_ARGUMENT, std::string("error writing ") + out_path);
}

int lbm_write_vtu(lbm_engine* e, const char* path, const int32_t cells[3]) {
    lbm::EngineView v;
    if (!e || !path || !cells || !lbm::engine_view(e, v)) return LBM_ERR_ARGUMENT;
    std::vector<double> rho(v.n), u(3 * v.n);
    if (int rc = lbm_get_macros(e, rho.data(), u.data())) return rc;
    // point order of WriteVTK_Collective: z outer, then y, x fastest
    std::vector<int64_t> ord(v.n);
    std::iota(ord.begin(), ord.end(), 0);
    const int32_t* c = v.coords;
    std::sort(ord.begin(), ord.end(), [c](int64_t a, int64_t b) {
        if (c[3 * a + 2] != c[3 * b + 2]) return c[3 * a + 2] < c[3 * b + 2];
        if (c[3 * a + 1] != c[3 * b + 1]) return c[3 * a + 1] < c[3 * b + 1];
        return c[3 * a] < c[3 * b];
    });
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t i = 0; i < v.n; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], c[3 * i + a]);
            hi[a] = std::max(hi[a], c[3 * i + a]);
        }
    const int64_t ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
    if ((double)ex * ey * ez > 4.0e9) return fail(LBM_ERR_ARGUMENT, "node set spans too large a box for the cell map");
    std::vector<int64_t> pid((size_t)(ex * ey * ez), -1);
    auto at = [&](int x, int y, int z) -> int64_t {
        if (x < lo[0] || y < lo[1] || z < lo[2] || x > hi[0] || y > hi[1] || z > hi[2]) return -1;
        return pid[((size_t)(x - lo[0]) * ey + (y - lo[1])) * ez + (z - lo[2])];
    };
    for (int64_t p = 0; p < v.n; ++p) {
        const int64_t i = ord[p];
        pid[((size_t)(c[3 * i] - lo[0]) * ey + (c[3 * i + 1] - lo[1])) * ez + (c[3 * i + 2] - lo[2])] = p;
    }
    std::vector<int64_t> conn;
    for (int z = 0; z < cells[2] - 1; ++z)
        for (int y = 0; y < cells[1] - 1; ++y)
            for (int x = 0; x < cells[0] - 1; ++x) {
                const int corner[8][3] = {{x, y, z},         {x + 1, y, z},         {x + 1, y + 1, z},
                                          {x, y + 1, z},     {x, y, z + 1},         {x + 1, y, z + 1},
                                          {x + 1, y + 1, z + 1}, {x, y + 1, z + 1}};
                int64_t ids[8];
                bool ok = true;
                for (int k = 0; k < 8 && ok; ++k) ok = (ids[k] = at(corner[k][0], corner[k][1], corner[k][2])) >= 0;
                if (ok) conn.insert(conn.end(), ids, ids + 8);
            }
    const int64_t nc = (int64_t)conn.size() / 8;
    std::vector<float> pts(3 * v.n);
    std::vector<double> vel(3 * v.n), den(v.n), mag(v.n);
    for (int64_t p = 0; p < v.n; ++p) {
        const int64_t i = ord[p];
        for (int a = 0; a < 3; ++a) {
            pts[3 * p + a] = (float)(double)c[3 * i + a];
            vel[3 * p + a] = u[3 * i + a];
        }
        den[p] = rho[i];
        const double* ui = &u[3 * i];
        mag[p] = std::sqrt(ui[0] * ui[0] + ui[1] * ui[1] + ui[2] * ui[2]);
    }
    std::vector<int64_t> offs(nc);
    for (int64_t k = 0; k < nc; ++k) offs[k] = 8 * (k + 1);
    std::vector<uint8_t> types(nc, 12);  // VTK_HEXAHEDRON
    struct Block {
        const void* p;
        uint64_t bytes;
    };
    const Block blocks[] = {{vel.data(), sizeof(double) * vel.size()}, {den.data(), sizeof(double) * den.size()},
                            {mag.data(), sizeof(double) * mag.size()}, {pts.data(), sizeof(float) * pts.size()},
                            {conn.data(), sizeof(int64_t) * conn.size()}, {offs.data(), sizeof(int64_t) * offs.size()},
                            {types.data(), types.size()}};
    uint64_t off[7], acc = 0;
    for (int b = 0; b < 7; ++b) {
        off[b] = acc;
        acc += 8 + blocks[b].bytes;
    }
    std::ofstream f(path, std::ios::binary);
    if (!f) return fail(LBM_ERR_ARGUMENT, std::string("cannot write ") + path);
    f << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
      << "  <UnstructuredGrid>\n"
      << "    <Piece NumberOfPoints=\"" << v.n << "\" NumberOfCells=\"" << nc << "\">\n"
      << "      <PointData>\n"
      << "        <DataArray type=\"Float64\" Name=\"Velocity\" NumberOfComponents=\"3\" format=\"appended\" offset=\""
      << off[0] << "\"/>\n"
      << "        <DataArray type=\"Float64\" Name=\"Density\" format=\"appended\" offset=\"" << off[1] << "\"/>\n"
      << "        <DataArray type=\"Float64\" Name=\"VelocityMagnitude\" format=\"appended\" offset=\"" << off[2]
      << "\"/>\n"
      << "      </PointData>\n"
      << "      <Points>\n"
      << "        <DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\" format=\"appended\" offset=\""
      << off[3] << "\"/>\n"
      << "      </Points>\n"
      << "      <Cells>\n"
      << "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"appended\" offset=\"" << off[4] << "\"/>\n"
      << "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"appended\" offset=\"" << off[5] << "\"/>\n"
      << "        <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"" << off[6] << "\"/>\n"
      << "      </Cells>\n"
      << "    </Piece>\n"
      << "  </UnstructuredGrid>\n"
      << "  <AppendedData encoding=\"raw\">\n   _";
    for (const Block& b : blocks) {
        f.write(reinterpret_cast<const char*>(&b.bytes), 8);
        if (b.bytes) f.write(static_cast<const char*>(b.p), (std::streamsize)b.bytes);
    }
    f << "\n  </AppendedData>\n</VTKFile>\n";
    return f.good() ? LBM_OK : fail(LBM_ERR_ARGUMENT, std::string("error writing ") + path);
}

}  // extern "C"
