// Stand-in for MadCart::CartesianMesh3D, the Cartesian grid STORM's examples use
// (MadCart is cloned unpinned by install_deps.sh:52 and is not available here).
// Written for this project: a rectilinear grid implementing exactly the Grid
// API STORM's hot path calls (GetPointNo, GetMeshPoint, GetCellFaces,
// GetFaceNeighbors, Normal, FaceCM, GetArea, GetVolume, GetBoxCoordinates,
// GetBoxFaces, IsPointOutsideBox, GetContainingCell, IsPointInCell,
// GetTotalFacesNumber, GetPointsInFace, GetFacePoints, GetBuildGeneration,
// GetCellCM).
//
// Conventions (the CUDA engine reproduces every one of them bit for bit):
//  * cell index            = i + nx*(j + ny*k)
//  * cell centre           = (0.5*(x_i + x_{i+1}), 0.5*(y_j + y_{j+1}), 0.5*(z_k + z_{k+1}))
//  * GetCellFaces(c) order = x-low, x-high, y-low, y-high, z-low, z-high
//  * face vertex order     = for a face normal to axis a with (b, c) the next
//                            axes cyclically (x->(y,z), y->(z,x), z->(x,y)):
//                            (b0,c0), (b1,c0), (b1,c1), (b0,c1)
//  * Normal(face)          = +unit vector of the face's axis
//  * ghost (outside) index = Ncells + global face index; its mesh point is the
//                            cell centre mirrored across the box face
//  * GetBoxFaces() order   = x-low, x-high, y-low, y-high, z-low, z-high with the
//                            same vertex order as cell faces
#ifndef STORM_SHIM_MADCART_CARTESIAN_MESH3D_HPP
#define STORM_SHIM_MADCART_CARTESIAN_MESH3D_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <utility>
#include <vector>

namespace MadCart {

template <typename PointT>
class CartesianMesh3D {
public:
    using Point_T = PointT;
    struct Face {
        std::vector<PointT> vertices;
    };
    using Face_T = Face;

    CartesianMesh3D(const PointT &ll, const PointT &ur, std::size_t nx, std::size_t ny, std::size_t nz)
        : CartesianMesh3D(uniform(ll.x, ur.x, nx), uniform(ll.y, ur.y, ny), uniform(ll.z, ur.z, nz)) {}

    CartesianMesh3D(const std::vector<double> &xEdges, double y0, double y1, std::size_t ny, double z0, double z1,
                    std::size_t nz)
        : CartesianMesh3D(xEdges, uniform(y0, y1, ny), uniform(z0, z1, nz)) {}

    CartesianMesh3D(const std::vector<double> &xe, const std::vector<double> &ye, const std::vector<double> &ze)
        : xe_(xe), ye_(ye), ze_(ze), generation_(nextGeneration()) {
        if (xe_.size() < 2 || ye_.size() < 2 || ze_.size() < 2) throw std::invalid_argument("CartesianMesh3D: need >= 1 cell per axis");
        nx_ = xe_.size() - 1;
        ny_ = ye_.size() - 1;
        nz_ = ze_.size() - 1;
        N_ = nx_ * ny_ * nz_;
        nxf_ = (nx_ + 1) * ny_ * nz_;
        nyf_ = nx_ * (ny_ + 1) * nz_;
        nzf_ = nx_ * ny_ * (nz_ + 1);
        build();
    }

    // A convex-polyhedral mesh in the box [lo, hi] (the stand-in for the
    // reference's Voronoi grids): per cell its faces, per face its neighbours
    // (the second >= N for a face on the box: the ghost N + f, whose mesh
    // point mirrors the cell's across that box plane), unit normal, centroid,
    // area and polygon.
    CartesianMesh3D(const PointT &lo, const PointT &hi, const std::vector<PointT> &points,
                    const std::vector<std::vector<std::size_t>> &cellFaces,
                    const std::vector<std::pair<std::size_t, std::size_t>> &faceNeighbors,
                    const std::vector<PointT> &normals, const std::vector<PointT> &faceCM,
                    const std::vector<double> &faceArea, const std::vector<double> &volume,
                    const std::vector<std::vector<std::size_t>> &faceVerts, const std::vector<PointT> &nodes)
        : xe_{lo.x, hi.x}, ye_{lo.y, hi.y}, ze_{lo.z, hi.z}, generation_(nextGeneration()), poly_(true) {
        N_ = points.size();
        nx_ = ny_ = nz_ = 0;
        points_ = points;
        cellFaces_ = cellFaces;
        faceNeighbors_ = faceNeighbors;
        normals_ = normals;
        faceCM_ = faceCM;
        faceArea_ = faceArea;
        volume_ = volume;
        faceVerts_ = faceVerts;
        nodes_ = nodes;
        points_.resize(N_ + faceNeighbors_.size());
        for (std::size_t f = 0; f < faceNeighbors_.size(); ++f) {
            const std::size_t g = faceNeighbors_[f].second;
            if (g < N_) continue;
            const PointT &c = faceCM_[f], &n = normals_[f];
            PointT m = points_[faceNeighbors_[f].first];
            // mirror across the box plane the face lies on
            if (std::abs(n.x) > 0.5) m.x = 2.0 * c.x - m.x;
            else if (std::abs(n.y) > 0.5) m.y = 2.0 * c.y - m.y;
            else m.z = 2.0 * c.z - m.z;
            points_[g] = m;
        }
        buildBoxFaces();
    }

    std::size_t GetPointNo() const { return N_; }
    const PointT &GetMeshPoint(std::size_t i) const { return points_[i]; }
    const PointT &GetCellCM(std::size_t i) const { return points_[i]; }
    const std::vector<std::size_t> &GetCellFaces(std::size_t c) const { return cellFaces_[c]; }
    const std::pair<std::size_t, std::size_t> &GetFaceNeighbors(std::size_t f) const { return faceNeighbors_[f]; }
    PointT Normal(std::size_t f) const {
        if (poly_) return normals_[f];
        int a = faceAxis(f);
        return PointT(a == 0 ? 1.0 : 0.0, a == 1 ? 1.0 : 0.0, a == 2 ? 1.0 : 0.0);
    }
    PointT FaceCM(std::size_t f) const { return faceCM_[f]; }
    double GetArea(std::size_t f) const { return faceArea_[f]; }
    double GetVolume(std::size_t c) const { return volume_[c]; }
    std::pair<PointT, PointT> GetBoxCoordinates() const {
        return {PointT(xe_.front(), ye_.front(), ze_.front()), PointT(xe_.back(), ye_.back(), ze_.back())};
    }
    const std::vector<Face_T> &GetBoxFaces() const { return boxFaces_; }
    bool IsPointOutsideBox(const PointT &p) const {
        return p.x < xe_.front() || p.x > xe_.back() || p.y < ye_.front() || p.y > ye_.back() ||
               p.z < ze_.front() || p.z > ze_.back();
    }
    bool IsPointOutsideBox(std::size_t index) const { return index >= N_; }
    std::size_t GetContainingCell(const PointT &p) const {
        if (poly_) {   // the nearest mesh point (Voronoi cells)
            std::size_t best = 0;
            double bd = 1e300;
            for (std::size_t c = 0; c < N_; ++c) {
                const double dx = p.x - points_[c].x, dy = p.y - points_[c].y, dz = p.z - points_[c].z;
                const double d = dx * dx + dy * dy + dz * dz;
                if (d < bd) { bd = d; best = c; }
            }
            return best;
        }
        std::size_t i = locate(xe_, p.x), j = locate(ye_, p.y), k = locate(ze_, p.z);
        return i + nx_ * (j + ny_ * k);
    }
    bool IsPointInCell(const PointT &p, std::size_t c) const {
        if (poly_) {
            for (std::size_t f : cellFaces_[c]) {
                PointT n = normals_[f];
                const PointT &q = faceCM_[f];
                const double side = n.x * (points_[c].x - q.x) + n.y * (points_[c].y - q.y) + n.z * (points_[c].z - q.z);
                const double d = n.x * (p.x - q.x) + n.y * (p.y - q.y) + n.z * (p.z - q.z);
                if ((side >= 0 ? d : -d) < 0) return false;
            }
            return true;
        }
        std::size_t i = c % nx_, j = (c / nx_) % ny_, k = c / (nx_ * ny_);
        return p.x >= xe_[i] && p.x <= xe_[i + 1] && p.y >= ye_[j] && p.y <= ye_[j + 1] && p.z >= ze_[k] &&
               p.z <= ze_[k + 1];
    }
    std::size_t GetTotalFacesNumber() const { return poly_ ? faceNeighbors_.size() : nxf_ + nyf_ + nzf_; }
    const std::vector<std::size_t> &GetPointsInFace(std::size_t f) const { return faceVerts_[f]; }
    const std::vector<PointT> &GetFacePoints() const { return nodes_; }
    // Unique per grid object: RandomPointOnFace (utils/RandomOnFace.hpp:20-33)
    // caches triangles keyed by (face, grid address, build generation), so two
    // grids that reuse one address must not share a generation.
    std::size_t GetBuildGeneration() const { return generation_; }

    std::size_t nx() const { return nx_; }
    std::size_t ny() const { return ny_; }
    std::size_t nz() const { return nz_; }

private:
    static std::size_t nextGeneration() {
        static std::size_t counter = 0;
        return ++counter;
    }
    static std::vector<double> uniform(double a, double b, std::size_t n) {
        std::vector<double> e(n + 1);
        for (std::size_t i = 0; i <= n; ++i) e[i] = a + (b - a) * static_cast<double>(i) / static_cast<double>(n);
        e[n] = b;
        return e;
    }
    std::size_t locate(const std::vector<double> &e, double v) const {
        std::size_t n = e.size() - 1;
        std::size_t idx = static_cast<std::size_t>(std::upper_bound(e.begin(), e.end(), v) - e.begin());
        if (idx == 0) return 0;
        idx -= 1;
        return idx >= n ? n - 1 : idx;
    }
    std::size_t node(std::size_t i, std::size_t j, std::size_t k) const { return i + (nx_ + 1) * (j + (ny_ + 1) * k); }
    int faceAxis(std::size_t f) const { return f < nxf_ ? 0 : (f < nxf_ + nyf_ ? 1 : 2); }
    std::size_t xFace(std::size_t i, std::size_t j, std::size_t k) const { return i + (nx_ + 1) * (j + ny_ * k); }
    std::size_t yFace(std::size_t i, std::size_t j, std::size_t k) const { return nxf_ + i + nx_ * (j + (ny_ + 1) * k); }
    std::size_t zFace(std::size_t i, std::size_t j, std::size_t k) const { return nxf_ + nyf_ + i + nx_ * (j + ny_ * k); }
    static double mid(double a, double b) { return 0.5 * (a + b); }

    void build() {
        nodes_.resize((nx_ + 1) * (ny_ + 1) * (nz_ + 1));
        for (std::size_t k = 0; k <= nz_; ++k)
            for (std::size_t j = 0; j <= ny_; ++j)
                for (std::size_t i = 0; i <= nx_; ++i) nodes_[node(i, j, k)] = PointT(xe_[i], ye_[j], ze_[k]);

        const std::size_t F = GetTotalFacesNumber();
        points_.assign(N_ + F, PointT(0.0, 0.0, 0.0));
        volume_.resize(N_);
        cellFaces_.resize(N_);
        faceNeighbors_.assign(F, {0, 0});
        faceCM_.resize(F);
        faceArea_.resize(F);
        faceVerts_.resize(F);

        for (std::size_t k = 0; k < nz_; ++k)
            for (std::size_t j = 0; j < ny_; ++j)
                for (std::size_t i = 0; i < nx_; ++i) {
                    std::size_t c = i + nx_ * (j + ny_ * k);
                    points_[c] = PointT(mid(xe_[i], xe_[i + 1]), mid(ye_[j], ye_[j + 1]), mid(ze_[k], ze_[k + 1]));
                    volume_[c] = (xe_[i + 1] - xe_[i]) * (ye_[j + 1] - ye_[j]) * (ze_[k + 1] - ze_[k]);
                    cellFaces_[c] = {xFace(i, j, k), xFace(i + 1, j, k), yFace(i, j, k), yFace(i, j + 1, k),
                                     zFace(i, j, k), zFace(i, j, k + 1)};
                }
        // x faces: (b, c) = (y, z)
        for (std::size_t k = 0; k < nz_; ++k)
            for (std::size_t j = 0; j < ny_; ++j)
                for (std::size_t i = 0; i <= nx_; ++i) {
                    std::size_t f = xFace(i, j, k);
                    faceVerts_[f] = {node(i, j, k), node(i, j + 1, k), node(i, j + 1, k + 1), node(i, j, k + 1)};
                    faceCM_[f] = PointT(xe_[i], mid(ye_[j], ye_[j + 1]), mid(ze_[k], ze_[k + 1]));
                    faceArea_[f] = (ye_[j + 1] - ye_[j]) * (ze_[k + 1] - ze_[k]);
                    link(f, i > 0 ? cellIdx(i - 1, j, k) : SIZE_MAX, i < nx_ ? cellIdx(i, j, k) : SIZE_MAX, 0, xe_[i]);
                }
        // y faces: (b, c) = (z, x)
        for (std::size_t k = 0; k < nz_; ++k)
            for (std::size_t j = 0; j <= ny_; ++j)
                for (std::size_t i = 0; i < nx_; ++i) {
                    std::size_t f = yFace(i, j, k);
                    faceVerts_[f] = {node(i, j, k), node(i, j, k + 1), node(i + 1, j, k + 1), node(i + 1, j, k)};
                    faceCM_[f] = PointT(mid(xe_[i], xe_[i + 1]), ye_[j], mid(ze_[k], ze_[k + 1]));
                    faceArea_[f] = (ze_[k + 1] - ze_[k]) * (xe_[i + 1] - xe_[i]);
                    link(f, j > 0 ? cellIdx(i, j - 1, k) : SIZE_MAX, j < ny_ ? cellIdx(i, j, k) : SIZE_MAX, 1, ye_[j]);
                }
        // z faces: (b, c) = (x, y)
        for (std::size_t k = 0; k <= nz_; ++k)
            for (std::size_t j = 0; j < ny_; ++j)
                for (std::size_t i = 0; i < nx_; ++i) {
                    std::size_t f = zFace(i, j, k);
                    faceVerts_[f] = {node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k)};
                    faceCM_[f] = PointT(mid(xe_[i], xe_[i + 1]), mid(ye_[j], ye_[j + 1]), ze_[k]);
                    faceArea_[f] = (xe_[i + 1] - xe_[i]) * (ye_[j + 1] - ye_[j]);
                    link(f, k > 0 ? cellIdx(i, j, k - 1) : SIZE_MAX, k < nz_ ? cellIdx(i, j, k) : SIZE_MAX, 2, ze_[k]);
                }
        // box faces
        const double X0 = xe_.front(), X1 = xe_.back(), Y0 = ye_.front(), Y1 = ye_.back(), Z0 = ze_.front(),
                     Z1 = ze_.back();
        (void)X0; (void)X1; (void)Y0; (void)Y1; (void)Z0; (void)Z1;
        buildBoxFaces();
    }
    void buildBoxFaces() {
        const double X0 = xe_.front(), X1 = xe_.back(), Y0 = ye_.front(), Y1 = ye_.back(), Z0 = ze_.front(),
                     Z1 = ze_.back();
        boxFaces_.resize(6);
        boxFaces_[0].vertices = {PointT(X0, Y0, Z0), PointT(X0, Y1, Z0), PointT(X0, Y1, Z1), PointT(X0, Y0, Z1)};
        boxFaces_[1].vertices = {PointT(X1, Y0, Z0), PointT(X1, Y1, Z0), PointT(X1, Y1, Z1), PointT(X1, Y0, Z1)};
        boxFaces_[2].vertices = {PointT(X0, Y0, Z0), PointT(X0, Y0, Z1), PointT(X1, Y0, Z1), PointT(X1, Y0, Z0)};
        boxFaces_[3].vertices = {PointT(X0, Y1, Z0), PointT(X0, Y1, Z1), PointT(X1, Y1, Z1), PointT(X1, Y1, Z0)};
        boxFaces_[4].vertices = {PointT(X0, Y0, Z0), PointT(X1, Y0, Z0), PointT(X1, Y1, Z0), PointT(X0, Y1, Z0)};
        boxFaces_[5].vertices = {PointT(X0, Y0, Z1), PointT(X1, Y0, Z1), PointT(X1, Y1, Z1), PointT(X0, Y1, Z1)};
    }
    std::size_t cellIdx(std::size_t i, std::size_t j, std::size_t k) const { return i + nx_ * (j + ny_ * k); }
    // Face neighbours (lower, upper); a missing side becomes the ghost N + f whose
    // mesh point mirrors the inside cell centre across the plane.
    void link(std::size_t f, std::size_t lo, std::size_t hi, int axis, double plane) {
        if (lo == SIZE_MAX || hi == SIZE_MAX) {
            std::size_t inside = (lo == SIZE_MAX) ? hi : lo;
            std::size_t ghost = N_ + f;
            PointT g = points_[inside];
            if (axis == 0) g.x = 2.0 * plane - g.x;
            if (axis == 1) g.y = 2.0 * plane - g.y;
            if (axis == 2) g.z = 2.0 * plane - g.z;
            points_[ghost] = g;
            if (lo == SIZE_MAX) lo = ghost; else hi = ghost;
        }
        faceNeighbors_[f] = {lo, hi};
    }

    std::vector<double> xe_, ye_, ze_;
    std::size_t generation_ = 0;
    bool poly_ = false;
    std::vector<PointT> normals_;
    std::size_t nx_ = 0, ny_ = 0, nz_ = 0, N_ = 0, nxf_ = 0, nyf_ = 0, nzf_ = 0;
    std::vector<PointT> nodes_, points_, faceCM_;
    std::vector<double> volume_, faceArea_;
    std::vector<std::vector<std::size_t>> cellFaces_, faceVerts_;
    std::vector<std::pair<std::size_t, std::size_t>> faceNeighbors_;
    std::vector<Face_T> boxFaces_;
};

} // namespace MadCart

#endif
