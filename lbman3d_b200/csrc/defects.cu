// defects.cu -- disclination lines from plaquette defect flags (host code):
// the connectivity graph and its path decomposition of the reference's
// DefectFinder (src/analysis/defect_finder.tpp:168-389,
// src/analysis/defect_connectivity_graph.h).
//
// Faces: def_x is nx x (ny-1) x (nz-1), def_y (nx-1) x ny x (nz-1), def_z
// (nx-1) x (ny-1) x nz, flattened x fastest; face ids are def_x, then def_y,
// then def_z (src/analysis/defect_fields.h:16-34).  Edges join flagged faces
// of one voxel and of the backward neighbours that the voxel sweep would
// otherwise miss, in the reference's sweep order (interior voxels, then the
// z, y and x boundary layers with the QXoff index clamp/wrap); the path
// decomposition walks the graph from the first odd-degree node (else the
// first node with an edge), always to the smallest neighbour, removing each
// edge it takes.  The graph is an unordered map of ordered neighbour sets,
// filled by the same sequence of insertions, so the walk visits nodes in the
// same order and yields the same disclinations as the reference's
// FindPaths.
#include <cstdint>
#include <cstring>
#include <optional>
#include <set>
#include <unordered_map>
#include <vector>

#include "../../include/lbman3d.h"

namespace lbman {
void set_last_error(const char* msg);
}

namespace {

using FaceId = std::uint64_t;

struct Faces {
    int nx, ny, nz;
    const uint8_t *fx, *fy, *fz;
    FaceId n_x, n_y;
    FaceId flat_x(int x, int y, int z) const { return (FaceId)(z * (ny - 1) + y) * (FaceId)nx + (FaceId)x; }
    FaceId flat_y(int x, int y, int z) const { return (FaceId)(z * ny + y) * (FaceId)(nx - 1) + (FaceId)x; }
    FaceId flat_z(int x, int y, int z) const { return (FaceId)(z * (ny - 1) + y) * (FaceId)(nx - 1) + (FaceId)x; }
    bool X(int x, int y, int z) const { return fx[flat_x(x, y, z)] == 1; }
    bool Y(int x, int y, int z) const { return fy[flat_y(x, y, z)] == 1; }
    bool Z(int x, int y, int z) const { return fz[flat_z(x, y, z)] == 1; }
    FaceId id_x(int x, int y, int z) const { return flat_x(x, y, z); }
    FaceId id_y(int x, int y, int z) const { return n_x + flat_y(x, y, z); }
    FaceId id_z(int x, int y, int z) const { return n_x + n_y + flat_z(x, y, z); }
    // face centre (src/analysis/defect_fields.h:74-101, unit spacing)
    void location(FaceId id, double* p) const {
        if (id >= n_x + n_y) {
            const FaceId i = id - n_x - n_y;
            const FaceId w = (FaceId)(nx - 1), h = (FaceId)(ny - 1);
            p[0] = (double)(i % w) + 0.5;
            p[1] = (double)((i / w) % h) + 0.5;
            p[2] = (double)(i / (w * h));
        } else if (id >= n_x) {
            const FaceId i = id - n_x;
            const FaceId w = (FaceId)(nx - 1), h = (FaceId)ny;
            p[0] = (double)(i % w) + 0.5;
            p[1] = (double)((i / w) % h);
            p[2] = (double)(i / (w * h)) + 0.5;
        } else {
            const FaceId w = (FaceId)nx, h = (FaceId)(ny - 1);
            p[0] = (double)(id % w);
            p[1] = (double)((id / w) % h) + 0.5;
            p[2] = (double)(id / (w * h)) + 0.5;
        }
    }
};

class Graph {
    std::unordered_map<FaceId, std::set<FaceId>> adj_;

public:
    void add(FaceId u, FaceId v) {
        if (u == v) return;
        adj_[u].insert(v);
        adj_[v].insert(u);
    }
    size_t edges() const {
        size_t n = 0;
        for (const auto& kv : adj_) n += kv.second.size();
        return n / 2;
    }
    std::optional<FaceId> start() const {
        for (const auto& kv : adj_)
            if (kv.second.size() % 2 == 1) return kv.first;
        for (const auto& kv : adj_)
            if (!kv.second.empty()) return kv.first;
        return std::nullopt;
    }
    std::vector<FaceId> walk(FaceId s) {
        std::vector<FaceId> path{s};
        while (true) {
            const FaceId u = path.back();
            auto& nu = adj_[u];
            if (nu.empty()) break;
            const FaceId v = *nu.begin();
            path.push_back(v);
            nu.erase(v);
            adj_[v].erase(u);
        }
        return path;
    }
};

// QAxisOffset (src/offsets.h:59-83): wrap on a Q-periodic face, clamp otherwise.
int qoff(int i, int s, int n, bool lo_periodic, bool hi_periodic) {
    const int j = i + s;
    if (j < 0) return lo_periodic ? ((j % n) + n) % n : 0;
    if (j >= n) return hi_periodic ? ((j % n) + n) % n : n - 1;
    return j;
}

void voxel(const Faces& F, Graph& g, int x, int y, int z, int xm, int xp, int ym, int yp, int zp) {
    const int nx = F.nx, ny = F.ny;
    if (F.X(x, y, z)) {
        const FaceId a = F.id_x(x, y, z);
        if (F.Z(x, y, z)) g.add(a, F.id_z(x, y, z));
        if (F.Z(x, y, zp)) g.add(a, F.id_z(x, y, zp));
        if (F.Y(x, y, z)) g.add(a, F.id_y(x, y, z));
        if (F.Y(x, yp, z)) g.add(a, F.id_y(x, yp, z));
        if (F.X(xp, y, z)) g.add(a, F.id_x(xp, y, z));
        if (xm < nx - 1 && F.Z(xm, y, zp)) g.add(a, F.id_z(xm, y, zp));
        if (xm < nx - 1 && F.Y(xm, yp, z)) g.add(a, F.id_y(xm, yp, z));
    }
    if (F.Y(x, y, z)) {
        const FaceId a = F.id_y(x, y, z);
        if (F.Z(x, y, z)) g.add(a, F.id_z(x, y, z));
        if (F.Z(x, y, zp)) g.add(a, F.id_z(x, y, zp));
        if (F.X(xp, y, z)) g.add(a, F.id_x(xp, y, z));
        if (F.Y(x, yp, z)) g.add(a, F.id_y(x, yp, z));
        if (ym < ny - 1 && F.Z(x, ym, zp)) g.add(a, F.id_z(x, ym, zp));
    }
    if (F.Z(x, y, z)) {
        const FaceId a = F.id_z(x, y, z);
        if (F.X(xp, y, z)) g.add(a, F.id_x(xp, y, z));
        if (F.Y(x, yp, z)) g.add(a, F.id_y(x, yp, z));
        if (F.Z(x, y, zp)) g.add(a, F.id_z(x, y, zp));
    }
}

}  // namespace

extern "C" int lbman_defect_graph(int nx, int ny, int nz, const int* qper6, const uint8_t* fx, const uint8_t* fy,
                                  const uint8_t* fz, lbman_defects* info, double* points, int64_t points_cap,
                                  int64_t* line_offsets, int64_t offsets_cap) {
    if (!qper6 || !fx || !fy || !fz || !info) {
        lbman::set_last_error("defect graph: null argument");
        return LBMAN_ERR_ARG;
    }
    if (nx < 2 || ny < 2 || nz < 2) {
        lbman::set_last_error("defect graph: every side must have at least 2 cells");
        return LBMAN_ERR_ARG;
    }
    const Faces F{nx, ny, nz, fx, fy, fz, (FaceId)nx * (ny - 1) * (nz - 1), (FaceId)(nx - 1) * ny * (nz - 1)};
    const FaceId n_z = (FaceId)(nx - 1) * (ny - 1) * nz;
    int64_t faces = 0;
    for (FaceId i = 0; i < F.n_x; ++i) faces += fx[i] == 1;
    for (FaceId i = 0; i < F.n_y; ++i) faces += fy[i] == 1;
    for (FaceId i = 0; i < n_z; ++i) faces += fz[i] == 1;
    Graph g;
    for (int z = 1; z < nz - 2; ++z)
        for (int y = 1; y < ny - 2; ++y)
            for (int x = 1; x < nx - 2; ++x) voxel(F, g, x, y, z, x - 1, x + 1, y - 1, y + 1, z + 1);
    auto edge_voxel = [&](int x, int y, int z) {
        voxel(F, g, x, y, z, qoff(x, -1, nx, qper6[0], qper6[1]), qoff(x, 1, nx, qper6[0], qper6[1]),
              qoff(y, -1, ny, qper6[2], qper6[3]), qoff(y, 1, ny, qper6[2], qper6[3]),
              qoff(z, 1, nz, qper6[4], qper6[5]));
    };
    for (int z : {0, nz - 2})
        for (int y = 0; y < ny - 1; ++y)
            for (int x = 0; x < nx - 1; ++x) edge_voxel(x, y, z);
    for (int z = 0; z < nz - 1; ++z)
        for (int y : {0, ny - 2})
            for (int x = 0; x < nx - 1; ++x) edge_voxel(x, y, z);
    for (int z = 0; z < nz - 1; ++z)
        for (int y = 0; y < ny - 1; ++y)
            for (int x : {0, nx - 2}) edge_voxel(x, y, z);
    info->faces = faces;
    info->edges = (int64_t)g.edges();
    int64_t nlines = 0, npts = 0;
    if (line_offsets && offsets_cap > 0) line_offsets[0] = 0;
    while (auto s = g.start()) {
        const std::vector<FaceId> path = g.walk(*s);
        for (FaceId id : path) {
            if (points && 3 * (npts + 1) <= points_cap) F.location(id, points + 3 * npts);
            ++npts;
        }
        ++nlines;
        if (line_offsets && nlines < offsets_cap) line_offsets[nlines] = npts;
    }
    info->lines = nlines;
    info->points = npts;
    return LBMAN_OK;
}
