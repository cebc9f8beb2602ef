// egt_knn_interface.hpp -- the reference's C++ class surface over the C ABI.
//
// The reference's consumers (EGT_CUDA, Normal_CUDA, getOutputPoints, main.cpp)
// are written against the abstract provider KNNInterface (KNNInterface.cuh:8-31)
// and the concrete providers GridStructure / GridMeshCuda.  This header keeps
// those names and call sequences, in namespace egtb200, on top of
// libegt_b200 (include/egt_b200.h), so code written like the reference's
// main.cpp:106-121 compiles against it with `using namespace egtb200;`.
// One GPU: num_cards must be 1.  Errors throw egtb200::Error.
#ifndef EGT_KNN_INTERFACE_HPP
#define EGT_KNN_INTERFACE_HPP

#include <cstdint>
#include <algorithm>
#include <stdexcept>
#include <string>
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

// Abstract provider, same getters as the reference's KNNInterface.cuh:8-31.
class KNNInterface {
public:
    virtual ~KNNInterface() = default;
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
};

// Provider backed by an egt_handle.  The device arrays behind the getters
// belong to the handle and are freed by the destructor, as in the reference
// (GridKNNCuda.cu:1005-1021).
class Provider : public KNNInterface {
public:
    explicit Provider(void* stream = nullptr) : stream_(stream) {}
    ~Provider() override { if (h_) egt_destroy(h_); }
    Provider(const Provider&) = delete;
    Provider& operator=(const Provider&) = delete;

    [[nodiscard]] bool isReady() const override { return views().lists != nullptr; }
    [[nodiscard]] int GetNumberOfCards() const override { return 1; }
    float** GetRefPointsX() override { refresh(); return &x_; }
    float** GetRefPointsY() override { refresh(); return &y_; }
    float** GetRefPointsZ() override { refresh(); return &z_; }
    int** GetKNNIndexesInPartitions() override { refresh(); return &lists_; }
    [[nodiscard]] int GetPartitionSize() const override { return (int)views().n; }
    int* GetPointCountInCards() override { refresh(); return &count_; }
    int** GetOriginalRefIndexes() override { refresh(); return &perm_; }
    void GetKNNIndexes(int* knn) override { check(egt_get_knn_host(h_, knn, stream_), "GetKNNIndexes"); }
    [[nodiscard]] float GetMaxExtent() const override { return views().max_extent; }
    [[nodiscard]] float GetMinExtent() const override { return views().min_extent; }
    [[nodiscard]] int pointsRefCount() const override { return (int)views().n; }
    [[nodiscard]] int NeighborCount() const override { return views().k; }

    egt_handle* handle() const { return h_; }
    void* stream() const { return stream_; }

protected:
    egt_views views() const {
        egt_views v{};
        check(egt_get_views(h_, &v), "egt_get_views");
        return v;
    }
    void refresh() {
        egt_views v = views();
        x_ = v.x; y_ = v.y; z_ = v.z; lists_ = v.lists; perm_ = v.perm; count_ = (int)v.n;
    }
    static egt_config make_config(float eps, int bucketCount) {
        egt_config c;
        egt_default_config(&c);
        c.eps = eps;
        c.bucket_count = bucketCount;
        return c;
    }
    egt_handle* h_ = nullptr;
    void* stream_ = nullptr;
    float *x_ = nullptr, *y_ = nullptr, *z_ = nullptr;
    int *lists_ = nullptr, *perm_ = nullptr;
    int count_ = 0;
};

// GridStructure(mesh, num_cards, eps, bucketCount, maxDivision) + GRIDCUDAKNNSELF_COMPACT.
// xyz: n points, AoS float (host memory), the layout of Mesh::mV.
class GridStructure : public Provider {
public:
    GridStructure(const float* xyz, int64_t n, int num_cards = 1, float eps = 1e-6f, int bucketCount = 1024,
                  int maxDivision = 4, void* stream = nullptr)
        : Provider(stream) {
        (void)maxDivision;  // the hierarchy always spans B = 1024 .. 8 (GridKNNCuda.cu:2464-2572)
        if (num_cards != 1) throw Error(EGT_ERR_ARG, "GridStructure: one GPU only (num_cards must be 1)");
        egt_config c = make_config(eps, bucketCount);
        check(egt_create_cloud(xyz, n, &c, stream_, &h_), "GridStructure");
        refresh();
    }
    void GRIDCUDAKNNSELF_COMPACT(int k, float thres = 1e8f) {
        if (thres != 1e8f) throw Error(EGT_ERR_ARG, "GRIDCUDAKNNSELF_COMPACT: thres is fixed at 1e8");
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
        if (thres != 1e8f) throw Error(EGT_ERR_ARG, "GRIDCUDAKNNCompact: thres is fixed at 1e8");
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
    std::vector<int> query_;
    int nq_ = -1, qk_ = 0;
};

// GridMeshCuda(mesh, num_cards, eps, bucketCount) + GetNeighborsFromTriangles.
class GridMeshCuda : public Provider {
public:
    GridMeshCuda(const float* xyz, int64_t n, const uint32_t* tris, int64_t t, int num_cards = 1,
                 float eps = 1e-6f, int bucketCount = 1024, void* stream = nullptr)
        : Provider(stream) {
        if (num_cards != 1) throw Error(EGT_ERR_ARG, "GridMeshCuda: one GPU only (num_cards must be 1)");
        egt_config c = make_config(eps, bucketCount);
        check(egt_create_mesh(xyz, n, tris, t, &c, stream_, &h_), "GridMeshCuda");
        refresh();
    }
    void GetNeighborsFromTriangles(int k) {
        check(egt_mesh_1ring(h_, k, stream_), "GetNeighborsFromTriangles");
        refresh();
    }
};

inline Provider& as_provider(KNNInterface& p) {
    auto* q = dynamic_cast<Provider*>(&p);
    if (!q) throw Error(EGT_ERR_ARG, "provider was not created by libegt_b200");
    return *q;
}

// EGT_CUDA(provider).PerformSmoothing(iterationCount, lambda, mu, alpha) (EGT_CUDA.cuh:11-46).
class EGT_CUDA {
public:
    explicit EGT_CUDA(KNNInterface& p) : p_(as_provider(p)) {}
    void PerformSmoothing(int iterationCount, float lambda = 0.63f, float mu = -0.64f, float alpha = 1e-8f) {
        check(egt_smooth(p_.handle(), iterationCount, lambda, mu, alpha, p_.stream()), "PerformSmoothing");
    }
private:
    Provider& p_;
};

// Normal_CUDA(provider).GetNormals(nx, ny, nz) (Normal_CUDA.cuh:10-25): host arrays, original order.
class Normal_CUDA {
public:
    explicit Normal_CUDA(KNNInterface& p) : p_(as_provider(p)) {}
    void GetNormals(float* nx, float* ny, float* nz) {
        check(egt_normals(p_.handle(), nx, ny, nz, p_.stream()), "GetNormals");
    }
private:
    Provider& p_;
};

// getOutputPoints(x, y, z, provider) (getOutputPoints.cuh:10): host arrays, original order.
inline void getOutputPoints(float* x, float* y, float* z, KNNInterface* p) {
    Provider& q = as_provider(*p);
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
