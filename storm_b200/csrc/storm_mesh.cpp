// Convex-polyhedral meshes for the engine: a bounded 3-D Voronoi tessellation
// of generator points in a box, in the face-list form the transport reads.
//
// Each cell starts as the box and is clipped by the bisector plane of its
// neighbours in order of distance (found through a uniform bin grid), until
// the next candidate is farther than twice the cell's farthest vertex, which
// no bisector beyond can cut.  A face shared by cells i < j is taken from
// cell i's polygon for both; a bisector face that only one side found (a
// sliver at rounding level) is added to the other side too, so adjacency is
// symmetric.  Box faces get ghost neighbours ncells + face index, as the
// reference's grids number cells outside the box.
//
// Face normals point from the face's first cell to its second; the transport
// turns them toward each cell's own mesh point.  Face centroids and areas come
// from a triangle fan of the ordered polygon; cell volumes from the fan
// tetrahedra of each face about the cell's mesh point (the decomposition the
// reference's RandomInCellPositionSampler draws positions from).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <thread>
#include <utility>
#include <vector>

#include "storm_cuda.h"

namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

// One face of a cell under construction: the plane n.x <= d bounds the cell,
// tag >= 0 is the neighbour cell, tag < 0 is box face -1 - tag.
struct PFace {
    V3 n;
    double d;
    int64_t tag;
    std::vector<V3> poly;   // counter-clockwise seen from outside (along n)
};

// Order points of a planar convex polygon counter-clockwise about normal n.
void order_polygon(std::vector<V3> &pts, V3 n) {
    if (pts.size() < 3) return;
    V3 c{0, 0, 0};
    for (auto &p : pts) c = c + p;
    c = c * (1.0 / pts.size());
    V3 a = std::fabs(n.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0};
    V3 u = cross(n, a);
    u = u * (1.0 / norm(u));
    V3 w = cross(n, u);
    std::vector<std::pair<double, V3>> ang;
    ang.reserve(pts.size());
    for (auto &p : pts) ang.push_back({std::atan2(dot(p - c, w), dot(p - c, u)), p});
    std::sort(ang.begin(), ang.end(), [](const std::pair<double, V3> &l, const std::pair<double, V3> &r) { return l.first < r.first; });
    pts.clear();
    for (auto &q : ang) pts.push_back(q.second);
}

// Clip the convex cell by n.x <= d; returns false when the plane does not cut it.
bool clip(std::vector<PFace> &cell, V3 n, double d, int64_t tag, double eps) {
    bool cuts = false;
    for (auto &f : cell)
        for (auto &v : f.poly)
            if (dot(n, v) - d > eps) { cuts = true; break; }
    if (!cuts) return false;
    std::vector<V3> cap;
    std::vector<PFace> out;
    out.reserve(cell.size() + 1);
    for (auto &f : cell) {
        std::vector<V3> np;
        const size_t m = f.poly.size();
        for (size_t k = 0; k < m; ++k) {
            const V3 a = f.poly[k], b = f.poly[(k + 1) % m];
            const double da = dot(n, a) - d, db = dot(n, b) - d;
            const bool ia = da <= eps, ib = db <= eps;
            if (ia) np.push_back(a);
            if (ia != ib) {
                const double t = da / (da - db);
                const V3 p = a + (b - a) * t;
                np.push_back(p);
                cap.push_back(p);
            } else if (ia && std::fabs(da) <= eps) {
                cap.push_back(a);
            }
        }
        if (np.size() >= 3) {
            f.poly.swap(np);
            out.push_back(std::move(f));
        }
    }
    // the new face: the cut's points, deduplicated and ordered
    std::vector<V3> uniq;
    for (auto &p : cap) {
        bool dup = false;
        for (auto &q : uniq)
            if (norm(p - q) <= 10 * eps) { dup = true; break; }
        if (!dup) uniq.push_back(p);
    }
    if (uniq.size() >= 3) {
        order_polygon(uniq, n);
        out.push_back(PFace{n, d, tag, std::move(uniq)});
    }
    cell.swap(out);
    return true;
}

double poly_area(const std::vector<V3> &p, V3 *cm) {
    V3 acc{0, 0, 0};
    double area = 0.0;
    for (size_t k = 1; k + 1 < p.size(); ++k) {
        const double a = 0.5 * norm(cross(p[k] - p[0], p[k + 1] - p[0]));
        acc = acc + (p[0] + p[k] + p[k + 1]) * (a / 3.0);
        area += a;
    }
    if (cm) *cm = area > 0.0 ? acc * (1.0 / area) : p[0];
    return area;
}

struct OwnedMesh : StormPolyMesh {
    std::vector<double> points, volume, faceNormal, faceCm, faceArea, vertices;
    std::vector<uint32_t> cellFaceOffset, cellFaces, faceCells, faceVertexOffset, faceVertices;
};

}  // namespace

extern "C" int storm_mesh_voronoi(const double *points, uint32_t n, const double box[6], StormPolyMesh **out) {
    if (!points || !box || !out || n == 0) return STORM_ERR_INVALID_ARG;
    const V3 lo{box[0], box[1], box[2]}, hi{box[3], box[4], box[5]};
    if (!(hi.x > lo.x && hi.y > lo.y && hi.z > lo.z)) return STORM_ERR_INVALID_ARG;
    std::vector<V3> P(n);
    for (uint32_t i = 0; i < n; ++i) {
        P[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        if (!(P[i].x > lo.x && P[i].x < hi.x && P[i].y > lo.y && P[i].y < hi.y && P[i].z > lo.z && P[i].z < hi.z))
            return STORM_ERR_INVALID_ARG;
    }
    const V3 ext = hi - lo;
    const double scale = std::max(ext.x, std::max(ext.y, ext.z));
    const double eps = 1e-13 * scale;
    // uniform bins, about 2 generators each
    const double h = std::cbrt(ext.x * ext.y * ext.z * 2.0 / n);
    const int bx = std::max(1, static_cast<int>(ext.x / h)), by = std::max(1, static_cast<int>(ext.y / h)),
              bz = std::max(1, static_cast<int>(ext.z / h));
    auto binOf = [&](V3 p, int &ix, int &iy, int &iz) {
        ix = std::min(bx - 1, std::max(0, static_cast<int>((p.x - lo.x) / ext.x * bx)));
        iy = std::min(by - 1, std::max(0, static_cast<int>((p.y - lo.y) / ext.y * by)));
        iz = std::min(bz - 1, std::max(0, static_cast<int>((p.z - lo.z) / ext.z * bz)));
    };
    std::vector<uint32_t> binStart(static_cast<size_t>(bx) * by * bz + 1, 0), binItems(n);
    {
        std::vector<uint32_t> cnt(static_cast<size_t>(bx) * by * bz, 0);
        std::vector<size_t> which(n);
        for (uint32_t i = 0; i < n; ++i) {
            int ix, iy, iz;
            binOf(P[i], ix, iy, iz);
            which[i] = (static_cast<size_t>(iz) * by + iy) * bx + ix;
            ++cnt[which[i]];
        }
        for (size_t b = 0; b < cnt.size(); ++b) binStart[b + 1] = binStart[b] + cnt[b];
        std::vector<uint32_t> fill(binStart.begin(), binStart.end() - 1);
        for (uint32_t i = 0; i < n; ++i) binItems[fill[which[i]]++] = i;
    }
    const double binW = std::min(ext.x / bx, std::min(ext.y / by, ext.z / bz));

    std::vector<std::vector<PFace>> cells(n);
    // cells are independent: host threads take interleaved indices
    auto buildCell = [&](uint32_t i) {
        std::vector<PFace> c;
        // the box: faces x-low, x-high, y-low, y-high, z-low, z-high (GetBoxFaces order)
        const V3 v[8] = {{lo.x, lo.y, lo.z}, {hi.x, lo.y, lo.z}, {hi.x, hi.y, lo.z}, {lo.x, hi.y, lo.z},
                         {lo.x, lo.y, hi.z}, {hi.x, lo.y, hi.z}, {hi.x, hi.y, hi.z}, {lo.x, hi.y, hi.z}};
        c.push_back({{-1, 0, 0}, -lo.x, -1, {v[0], v[4], v[7], v[3]}});
        c.push_back({{1, 0, 0}, hi.x, -2, {v[1], v[2], v[6], v[5]}});
        c.push_back({{0, -1, 0}, -lo.y, -3, {v[0], v[1], v[5], v[4]}});
        c.push_back({{0, 1, 0}, hi.y, -4, {v[3], v[7], v[6], v[2]}});
        c.push_back({{0, 0, -1}, -lo.z, -5, {v[0], v[3], v[2], v[1]}});
        c.push_back({{0, 0, 1}, hi.z, -6, {v[4], v[5], v[6], v[7]}});
        int ix, iy, iz;
        binOf(P[i], ix, iy, iz);
        std::vector<std::pair<double, uint32_t>> cand;
        int ring = 0;
        size_t done = 0;   // candidates already used
        for (;;) {
            // candidates in the shell of bins at Chebyshev distance `ring`
            for (int z = iz - ring; z <= iz + ring; ++z)
                for (int y = iy - ring; y <= iy + ring; ++y)
                    for (int x = ix - ring; x <= ix + ring; ++x) {
                        if (std::max(std::abs(x - ix), std::max(std::abs(y - iy), std::abs(z - iz))) != ring) continue;
                        if (x < 0 || y < 0 || z < 0 || x >= bx || y >= by || z >= bz) continue;
                        const size_t b = (static_cast<size_t>(z) * by + y) * bx + x;
                        for (uint32_t q = binStart[b]; q < binStart[b + 1]; ++q) {
                            const uint32_t j = binItems[q];
                            if (j != i) cand.push_back({norm(P[j] - P[i]), j});
                        }
                    }
            std::sort(cand.begin() + done, cand.end());
            // every generator closer than `ring * binW` has been seen
            const double safe = ring * binW;
            double rmax = 0.0;
            for (auto &f : c)
                for (auto &vv : f.poly) rmax = std::max(rmax, norm(vv - P[i]));
            while (done < cand.size() && cand[done].first <= safe) {
                if (cand[done].first > 2.0 * rmax) break;
                const uint32_t j = cand[done].second;
                const V3 nn = (P[j] - P[i]) * (1.0 / cand[done].first);
                const double d = dot(nn, (P[i] + P[j]) * 0.5);
                if (clip(c, nn, d, j, eps)) {
                    rmax = 0.0;
                    for (auto &f : c)
                        for (auto &vv : f.poly) rmax = std::max(rmax, norm(vv - P[i]));
                }
                ++done;
            }
            const bool exhausted = ring > std::max(bx, std::max(by, bz));
            if (exhausted || 2.0 * rmax < safe) break;
            ++ring;
        }
        cells[i].swap(c);
    };
    {
        unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        if (n < 4096) nt = 1;
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t)
            pool.emplace_back([&, t] {
                for (uint32_t i = t; i < n; i += nt) buildCell(i);
            });
        for (auto &th : pool) th.join();
    }

    // global faces
    auto *om = new (std::nothrow) OwnedMesh();
    if (!om) return STORM_ERR_OOM;
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> pairFace;
    std::vector<std::vector<uint32_t>> cellF(n);
    auto addFace = [&](uint32_t a, uint32_t bNeighbor, bool ghost, const std::vector<V3> &poly, V3 nrm) {
        const uint32_t f = static_cast<uint32_t>(om->faceArea.size());
        V3 cm;
        const double area = poly_area(poly, &cm);
        om->faceCells.push_back(a);
        om->faceCells.push_back(ghost ? n + f : bNeighbor);
        om->faceNormal.insert(om->faceNormal.end(), {nrm.x, nrm.y, nrm.z});
        om->faceCm.insert(om->faceCm.end(), {cm.x, cm.y, cm.z});
        om->faceArea.push_back(area);
        om->faceVertexOffset.push_back(static_cast<uint32_t>(om->vertices.size() / 3));
        for (auto &p : poly) om->vertices.insert(om->vertices.end(), {p.x, p.y, p.z});
        return f;
    };
    om->faceVertexOffset.clear();
    for (uint32_t i = 0; i < n; ++i) {
        for (auto &f : cells[i]) {
            if (f.tag < 0) {
                cellF[i].push_back(addFace(i, 0, true, f.poly, f.n));
            } else {
                const uint32_t j = static_cast<uint32_t>(f.tag);
                const auto key = std::make_pair(std::min(i, j), std::max(i, j));
                auto it = pairFace.find(key);
                if (it == pairFace.end()) {
                    // first seen from cell i: normal from the lower cell to the higher one
                    const uint32_t a = key.first, b = key.second;
                    V3 nrm = P[b] - P[a];
                    nrm = nrm * (1.0 / norm(nrm));
                    std::vector<V3> poly = f.poly;
                    if (a != i) std::reverse(poly.begin(), poly.end());
                    const uint32_t gf = addFace(a, b, false, poly, nrm);
                    pairFace[key] = gf;
                    cellF[i].push_back(gf);
                } else {
                    cellF[i].push_back(it->second);
                }
            }
        }
    }
    // symmetric adjacency: a face only one side found is added to the other side
    for (auto &kv : pairFace) {
        const uint32_t a = kv.first.first, b = kv.first.second, f = kv.second;
        for (uint32_t c : {a, b})
            if (std::find(cellF[c].begin(), cellF[c].end(), f) == cellF[c].end()) cellF[c].push_back(f);
    }
    const uint32_t F = static_cast<uint32_t>(om->faceArea.size());
    om->faceVertexOffset.push_back(static_cast<uint32_t>(om->vertices.size() / 3));
    for (uint32_t v = 0; v < om->vertices.size() / 3; ++v) om->faceVertices.push_back(v);
    om->cellFaceOffset.assign(1, 0);
    for (uint32_t i = 0; i < n; ++i) {
        om->cellFaces.insert(om->cellFaces.end(), cellF[i].begin(), cellF[i].end());
        om->cellFaceOffset.push_back(static_cast<uint32_t>(om->cellFaces.size()));
    }
    om->points.assign(points, points + 3 * static_cast<size_t>(n));
    om->volume.assign(n, 0.0);
    for (uint32_t i = 0; i < n; ++i) {
        double vol = 0.0;
        for (uint32_t f : cellF[i]) {
            const uint32_t v0 = om->faceVertexOffset[f], v1 = om->faceVertexOffset[f + 1];
            if (v1 - v0 < 3) continue;
            auto vert = [&](uint32_t k) { return V3{om->vertices[3 * k], om->vertices[3 * k + 1], om->vertices[3 * k + 2]}; };
            for (uint32_t k = v0 + 1; k + 1 < v1; ++k) {
                const V3 a = vert(v0) - P[i], b = vert(k) - P[i], c = vert(k + 1) - P[i];
                vol += std::fabs(dot(a, cross(b, c)));
            }
        }
        om->volume[i] = vol / 6.0;
    }
    StormPolyMesh &m = *om;
    m.ncells = n;
    m.nfaces = F;
    m.nvertices = static_cast<uint32_t>(om->vertices.size() / 3);
    for (int k = 0; k < 6; ++k) m.box[k] = box[k];
    m.points = om->points.data();
    m.volume = om->volume.data();
    m.cell_face_offset = om->cellFaceOffset.data();
    m.cell_faces = om->cellFaces.data();
    m.face_cells = om->faceCells.data();
    m.face_normal = om->faceNormal.data();
    m.face_cm = om->faceCm.data();
    m.face_area = om->faceArea.data();
    m.face_vertex_offset = om->faceVertexOffset.data();
    m.face_vertices = om->faceVertices.data();
    m.vertices = om->vertices.data();
    *out = &m;
    return STORM_OK;
}

extern "C" int storm_mesh_free(StormPolyMesh *m) {
    if (!m) return STORM_OK;
    delete static_cast<OwnedMesh *>(m);
    return STORM_OK;
}
