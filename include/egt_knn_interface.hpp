// egt_knn_interface.hpp -- the reference's C++ class surface over the C ABI.
//
// The reference's consumers (EGT_CUDA, Normal_CUDA, getOutputPoints, main.cpp)
// are written against the abstract provider KNNInterface (KNNInterface.cuh:8-31)
// and the concrete providers GridStructure / GridMeshCuda.  This header keeps
// those names and call sequences, in namespace egtb200, on top of
// libegt_b200 (include/egt_b200.h), so code written like the reference's
// main.cpp:106-121 compiles against it with `using namespace egtb200;`.
// One GPU: num_cards must be 1.  Errors throw egtb200::Error.
//
// Slots.  As in the reference, the getters GetRefPointsX/Y/Z() and
// GetKNNIndexesInPartitions() return the address of a one-entry slot array
// holding a device pointer, and a consumer may write through that pointer (the
// EGT filter writes -1 into the lists, EGT_CUDA.cu:172-189) or swap a buffer of
// its own into the slot (EGT_CUDA.cu:591-596).  The slots keep whatever the
// consumer left; before any stage of this library runs on the provider, what
// the slots hold is handed back to the handle (egt_commit_views), and a buffer a
// consumer swapped in is then released, as the reference's destructor frees
// whatever its slots hold (GridKNNCuda.cu:1005-1021).
//
// Code compiled against the reference's own KNNInterface.cuh takes these
// providers through ReferenceView<::KNNInterface> (below).
#ifndef EGT_KNN_INTERFACE_HPP
#define EGT_KNN_INTERFACE_HPP

#include <cstdint>
#include <algorithm>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "egt_b200.h"

namespace egtb200 {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(egt_status s, const char* what) {
    if (s != EGT_OK) throw Error(s, std::string(what) + ": " + egt_last_error());
}

// Abstract provider, the same virtual getters in the same order as the
// reference's KNNInterface.cuh:8-31 (and, like it, no virtual destructor).
class KNNInterface {
public:
    [[nodiscard]] virtual bool isReady() const = 0;
    [[nodiscard]] virtual int GetNumberOfCards() const = 0;
    virtual float** GetRefPointsX() = 0;
    virtual float** GetRefPointsY() = 0;
    virtual float** GetRefPointsZ() = 0;
    virtual float** GetQuerPointsX() { return GetRefPointsX(); }
    virtual float** GetQuerPointsY() { return GetRefPointsY(); }
    virtual float** GetQuerPointsZ() { return GetRefPointsZ(); }
    virtual int** GetKNNIndexesInPartitions() = 0;
    [[nodiscard]] virtual int GetPartitionSize() const = 0;
    virtual int* GetPointCountInCards() = 0;
    virtual int** GetOriginalRefIndexes() = 0;
    virtual int** GetOriginalQuerIndexes() { return GetOriginalRefIndexes(); }
    virtual void GetKNNIndexes(int* knnIndexes) = 0;
    [[nodiscard]] virtual float GetMaxExtent() const = 0;
    [[nodiscard]] virtual float GetMinExtent() const = 0;
    [[nodiscard]] virtual int pointsRefCount() const = 0;
    [[nodiscard]] virtual int pointsQuerCount() const { return pointsRefCount(); }
    [[nodiscard]] virtual int NeighborCount() const = 0;

protected:
    ~KNNInterface() = default;
};

// Provider backed by an egt_handle.  The device arrays behind the getters
// belong to the handle and are freed by the destructor, as in the reference
// (GridKNNCuda.cu:1005-1021).
class Provider : public KNNInterface {
public:
    explicit Provider(void* stream = nullptr) : stream_(stream) {}
    virtual ~Provider() {
        if (!h_) return;
        egt_views v{};
        if (egt_get_views(h_, &v) == EGT_OK) release_foreign(v);
        egt_destroy(h_);
    }
    Provider(const Provider&) = delete;
    Provider& operator=(const Provider&) = delete;

    [[nodiscard]] bool isReady() const override { return lists_ != nullptr; }
    [[nodiscard]] int GetNumberOfCards() const override { return 1; }
    float** GetRefPointsX() override { lent_ = true; return &x_; }
    float** GetRefPointsY() override { lent_ = true; return &y_; }
    float** GetRefPointsZ() override { lent_ = true; return &z_; }
    int** GetKNNIndexesInPartitions() override { lent_ = true; return &lists_; }
    [[nodiscard]] int GetPartitionSize() const override { return count_; }
    int* GetPointCountInCards() override { return &count_; }
    int** GetOriginalRefIndexes() override { return &perm_; }
    void GetKNNIndexes(int* knn) override {
        sync();
        check(egt_get_knn_host(h_, knn, stream_), "GetKNNIndexes");
    }
    [[nodiscard]] float GetMaxExtent() const override { return max_; }
    [[nodiscard]] float GetMinExtent() const override { return min_; }
    [[nodiscard]] int pointsRefCount() const override { return count_; }
    [[nodiscard]] int NeighborCount() const override { return k_; }

    egt_handle* handle() const { return h_; }
    void* stream() const { return stream_; }

    // Hands what a consumer left in the slots back to the handle (called
    // before every stage of this library that runs on this provider).
    void sync() {
        if (!lent_) return;
        lent_ = false;
        check(egt_commit_views(h_, x_, y_, z_, stream_), "egt_commit_views");
        egt_views v = views();
        release_foreign(v);
        if (lists_ != v.lists)  // the reference's consumers write the lists in place, never swap them
            throw Error(EGT_ERR_ARG, "a consumer replaced the list buffer; write the lists in place instead");
        refresh();
    }
    // Re-reads the slots from the handle after a stage of this library.
    void refresh() {
        egt_views v = views();
        x_ = v.x; y_ = v.y; z_ = v.z; lists_ = v.lists; perm_ = v.perm;
        count_ = (int)v.n;
        k_ = v.k;
        min_ = v.min_extent;
        max_ = v.max_extent;
    }

protected:
    egt_views views() const {
        egt_views v{};
        check(egt_get_views(h_, &v), "egt_get_views");
        return v;
    }
    // Frees position buffers a consumer swapped into the slots (the handle's
    // own arrays are freed with the handle).
    void release_foreign(const egt_views& v) {
        if (x_ && x_ != v.x) egt_free_device(x_);
        if (y_ && y_ != v.y) egt_free_device(y_);
        if (z_ && z_ != v.z) egt_free_device(z_);
        x_ = v.x; y_ = v.y; z_ = v.z;
    }
    static egt_config make_config(float eps, int bucketCount) {
        egt_config c;
        egt_default_config(&c);
        c.eps = eps;
        c.bucket_count = bucketCount;
        return c;
    }
    // The reference builds its cell hierarchy down to B = maxDivision
    // (GridKNNCuda.cu:1196-1204) while its search descends to B = 8 (:2464-2572);
    // a query that needs a level it did not build reads past its hierarchy
    // (InitializeLevel, :937-946).  This library always builds B = 1024..8, so
    // its lists equal the reference's wherever those are defined, for every
    // maxDivision >= 1.
    static void check_division(int maxDivision) {
        if (maxDivision < 1) throw Error(EGT_ERR_ARG, "maxDivision must be >= 1");
    }
    // thres of the reference's searches (GridKNNCuda.cu:2324-2325), set on the
    // handle when it changes.
    void use_threshold(float thres) {
        if (thres != thres_) {
            check(egt_set_threshold(h_, thres, stream_), "threshold");
            thres_ = thres;
        }
    }
    egt_handle* h_ = nullptr;
    void* stream_ = nullptr;
    float *x_ = nullptr, *y_ = nullptr, *z_ = nullptr;
    int *lists_ = nullptr, *perm_ = nullptr;
    int count_ = 0, k_ = 0;
    float min_ = 0.0f, max_ = 0.0f, thres_ = 1e8f;
    bool lent_ = false;
};

// GridStructure(mesh, num_cards, eps, bucketCount, maxDivision) + its searches.
class GridStructure : public Provider {
public:
    // The reference's constructor: any mesh type with the layout of Mesh.h's
    // Mesh (a std::vector mV of {float x, y, z}).
    template <class MeshT, class = decltype(std::declval<const MeshT&>().mV.data()->x)>
    GridStructure(const MeshT& mesh, int num_cards, float eps = 1e-6f, int bucketCount = 1024,
                  int maxDivision = 32, void* stream = nullptr)
        : GridStructure(points_of(mesh), (int64_t)mesh.mV.size(), num_cards, eps, bucketCount, maxDivision, stream) {}
    // xyz: n points, AoS float (host memory), the layout of Mesh::mV.
    GridStructure(const float* xyz, int64_t n, int num_cards = 1, float eps = 1e-6f, int bucketCount = 1024,
                  int maxDivision = 32, void* stream = nullptr)
        : Provider(stream) {
        check_division(maxDivision);
        if (num_cards != 1) throw Error(EGT_ERR_ARG, "GridStructure: one GPU only (num_cards must be 1)");
        egt_config c = make_config(eps, bucketCount);
        check(egt_create_cloud(xyz, n, &c, stream_, &h_), "GridStructure");
        refresh();
    }
    void GRIDCUDAKNNSELF_COMPACT(int k, float thres = 1e8f) {
        sync();
        use_threshold(thres);
        check(egt_knn(h_, k, stream_), "GRIDCUDAKNNSELF_COMPACT");
        query_.clear();
        nq_ = -1;
        refresh();
    }
    // GridStructure::GRIDCUDAKNNCompact (GridKNNCuda.cu:1645-1939): the k
    // nearest reference points of nq query points (host SoA, the reference's
    // units).  As in the reference, GetKNNIndexes then returns the query
    // lists (nq rows in query order) until the next self search.
    void GRIDCUDAKNNCompact(const float* qx, const float* qy, const float* qz, int nq, int k, float thres = 1e8f) {
        sync();
        use_threshold(thres);
        std::vector<float> q(3 * (size_t)nq);
        for (int i = 0; i < nq; i++) {
            q[3 * (size_t)i] = qx[i];
            q[3 * (size_t)i + 1] = qy[i];
            q[3 * (size_t)i + 2] = qz[i];
        }
        query_.assign((size_t)nq * k, -1);
        check(egt_knn_query(h_, q.data(), nq, k, query_.data(), nullptr, stream_), "GRIDCUDAKNNCompact");
        nq_ = nq;
        qk_ = k;
    }
    void GetKNNIndexes(int* knn) override {
        if (nq_ < 0) return Provider::GetKNNIndexes(knn);
        std::copy(query_.begin(), query_.end(), knn);
    }
    [[nodiscard]] int pointsQuerCount() const override { return nq_ < 0 ? pointsRefCount() : nq_; }
    [[nodiscard]] int NeighborCount() const override { return nq_ < 0 ? Provider::NeighborCount() : qk_; }

private:
    template <class MeshT>
    static const float* points_of(const MeshT& mesh) {
        static_assert(sizeof(*mesh.mV.data()) == 3 * sizeof(float), "Mesh::mV must hold {float x, y, z}");
        return reinterpret_cast<const float*>(mesh.mV.data());
    }
    std::vector<int> query_;
    int nq_ = -1, qk_ = 0;
};

// GridMeshCuda(mesh, num_cards, eps, bucketCount) + GetNeighborsFromTriangles.
class GridMeshCuda : public Provider {
public:
    // The reference's constructor: a mesh with Mesh.h's layout (mV of
    // {float x, y, z}, mF of {uint32_t v0, v1, v2}).
    template <class MeshT, class = decltype(std::declval<const MeshT&>().mF.data()->v0)>
    GridMeshCuda(const MeshT& mesh, int num_cards, float eps = 1e-6f, int bucketCount = 1024, void* stream = nullptr)
        : GridMeshCuda(points_of(mesh), (int64_t)mesh.mV.size(), faces_of(mesh), (int64_t)mesh.mF.size(), num_cards,
                       eps, bucketCount, stream) {}
    GridMeshCuda(const float* xyz, int64_t n, const uint32_t* tris, int64_t t, int num_cards = 1,
                 float eps = 1e-6f, int bucketCount = 1024, void* stream = nullptr)
        : Provider(stream) {
        if (num_cards != 1) throw Error(EGT_ERR_ARG, "GridMeshCuda: one GPU only (num_cards must be 1)");
        egt_config c = make_config(eps, bucketCount);
        check(egt_create_mesh(xyz, n, tris, t, &c, stream_, &h_), "GridMeshCuda");
        refresh();
    }
    void GetNeighborsFromTriangles(int k) {
        sync();
        check(egt_mesh_1ring(h_, k, stream_), "GetNeighborsFromTriangles");
        refresh();
    }

private:
    template <class MeshT>
    static const float* points_of(const MeshT& mesh) {
        static_assert(sizeof(*mesh.mV.data()) == 3 * sizeof(float), "Mesh::mV must hold {float x, y, z}");
        return reinterpret_cast<const float*>(mesh.mV.data());
    }
    template <class MeshT>
    static const uint32_t* faces_of(const MeshT& mesh) {
        static_assert(sizeof(*mesh.mF.data()) == 3 * sizeof(uint32_t), "Mesh::mF must hold {uint32_t v0, v1, v2}");
        return reinterpret_cast<const uint32_t*>(mesh.mF.data());
    }
};

inline Provider& as_provider(KNNInterface& p) {
    auto* q = dynamic_cast<Provider*>(&p);
    if (!q) throw Error(EGT_ERR_ARG, "provider was not created by libegt_b200");
    return *q;
}

// A provider as seen by code compiled against the reference's own
// KNNInterface.cuh (the reference's EGT_CUDA, Normal_CUDA, getOutputPoints):
//     egtb200::GridStructure grid(mesh, 1, 1e-6, 1024, 4);
//     grid.GRIDCUDAKNNSELF_COMPACT(k, 1e8);
//     egtb200::ReferenceView<::KNNInterface> view(grid);
//     EGT_CUDA smoother(view);              // the reference's class
// The view's getters are the provider's own slots, so what a reference
// consumer writes or swaps there is seen by the provider (and handed to the
// handle before the provider's next stage).  The view must not outlive it.
template <class Base>
class ReferenceView : public Base {
public:
    explicit ReferenceView(Provider& p) : p_(p) {}
    [[nodiscard]] bool isReady() const override { return p_.isReady(); }
    [[nodiscard]] int GetNumberOfCards() const override { return 1; }
    float** GetRefPointsX() override { return p_.GetRefPointsX(); }
    float** GetRefPointsY() override { return p_.GetRefPointsY(); }
    float** GetRefPointsZ() override { return p_.GetRefPointsZ(); }
    float** GetQuerPointsX() override { return p_.GetQuerPointsX(); }
    float** GetQuerPointsY() override { return p_.GetQuerPointsY(); }
    float** GetQuerPointsZ() override { return p_.GetQuerPointsZ(); }
    int** GetKNNIndexesInPartitions() override { return p_.GetKNNIndexesInPartitions(); }
    [[nodiscard]] int GetPartitionSize() const override { return p_.GetPartitionSize(); }
    int* GetPointCountInCards() override { return p_.GetPointCountInCards(); }
    int** GetOriginalRefIndexes() override { return p_.GetOriginalRefIndexes(); }
    int** GetOriginalQuerIndexes() override { return p_.GetOriginalQuerIndexes(); }
    void GetKNNIndexes(int* knnIndexes) override { p_.GetKNNIndexes(knnIndexes); }
    [[nodiscard]] float GetMaxExtent() const override { return p_.GetMaxExtent(); }
    [[nodiscard]] float GetMinExtent() const override { return p_.GetMinExtent(); }
    [[nodiscard]] int pointsRefCount() const override { return p_.pointsRefCount(); }
    [[nodiscard]] int pointsQuerCount() const override { return p_.pointsQuerCount(); }
    [[nodiscard]] int NeighborCount() const override { return p_.NeighborCount(); }

private:
    Provider& p_;
};

// EGT_CUDA(provider).PerformSmoothing(iterationCount, lambda, mu, alpha) (EGT_CUDA.cuh:11-46).
class EGT_CUDA {
public:
    explicit EGT_CUDA(KNNInterface& p) : p_(as_provider(p)) {}
    void PerformSmoothing(int iterationCount, float lambda = 0.63f, float mu = -0.64f, float alpha = 1e-8f) {
        p_.sync();
        check(egt_smooth(p_.handle(), iterationCount, lambda, mu, alpha, p_.stream()), "PerformSmoothing");
        p_.refresh();
    }
private:
    Provider& p_;
};

// Normal_CUDA(provider).GetNormals(nx, ny, nz) (Normal_CUDA.cuh:10-25): host arrays, original order.
class Normal_CUDA {
public:
    explicit Normal_CUDA(KNNInterface& p) : p_(as_provider(p)) {}
    void GetNormals(float* nx, float* ny, float* nz) {
        p_.sync();
        check(egt_normals(p_.handle(), nx, ny, nz, p_.stream()), "GetNormals");
    }
private:
    Provider& p_;
};

// getOutputPoints(x, y, z, provider) (getOutputPoints.cuh:10): host arrays, original order.
inline void getOutputPoints(float* x, float* y, float* z, KNNInterface* p) {
    Provider& q = as_provider(*p);
    q.sync();
    check(egt_output(q.handle(), x, y, z, q.stream()), "getOutputPoints");
}

// orient_kruskal(knn, nx, ny, nz, x, y, z, N, k, k_use) (MST.h:11-12,
// MST.cpp:399-423): the reference's CPU orienter, same signature, computed on
// GPU 0 with the same oriented normals (see egt_orient_kruskal).
inline void orient_kruskal(int* knn, float* nx, float* ny, float* nz, float* x, float* y, float* z, int N, int k,
                           int k_use) {
    check(egt_orient_kruskal(knn, nx, ny, nz, x, y, z, N, k, k_use, 0, nullptr), "orient_kruskal");
}

}  // namespace egtb200

#endif  // EGT_KNN_INTERFACE_HPP
