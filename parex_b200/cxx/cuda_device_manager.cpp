// Drop-in implementation of the reference's CudaDeviceManager
// (cuda/interface.h:16-57) on top of the parex_b200 C ABI.
//
// Compiled against the reference's own headers (cuda/interface.h,
// lib/core/graph.h, lib/core/definitions.h) so that the class layout and the
// mangled member names are the reference's; an application such as the
// reference's main.cpp relinks against this file and libparex_b200.so
// unchanged.  Like the reference, the seed and both thresholds are read from
// the globals randSeed, sc_threshold and rw_threshold when initialize() runs
// (lib/core/definitions.h:46-50).  Unlike the reference, failures do not pass
// silently: a failing call throws std::runtime_error with the library's
// message.
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "cuda/interface.h"
#include "parex_b200.h"

struct CudaDeviceManager::Impl {
    pxr_handle* h = nullptr;
    NodeIx n = 0;
    EdgeIx m = 0;

    ~Impl() { reset(); }

    void reset() {
        if (h) pxr_destroy(h);
        h = nullptr;
    }

    void check(pxr_status s, const char* what) const {
        if (s != PXR_OK)
            throw std::runtime_error(std::string("parex_b200: ") + what + ": " + pxr_status_string(s) + ": " +
                                     (h ? pxr_last_error(h) : ""));
    }

    pxr_handle* need() const {
        if (!h) throw std::runtime_error("parex_b200: initialize() has not been called");
        return h;
    }
};

CudaDeviceManager::CudaDeviceManager() : impl(std::make_unique<Impl>()) {}

CudaDeviceManager::~CudaDeviceManager() = default;

void CudaDeviceManager::initialize(const Graph& graph) {
    impl->reset();
    pxr_config cfg;
    pxr_config_default(&cfg);
    cfg.seed = randSeed;
    cfg.sc_threshold = sc_threshold;
    cfg.rw_threshold = rw_threshold;
    impl->check(pxr_create(&cfg, &impl->h), "pxr_create");
    impl->n = graph.numNodes;
    impl->m = graph.numEdges;
    impl->check(pxr_initialize(impl->h, graph.numNodes, graph.numEdges, graph.ranges.data(), graph.edges.data()),
                "initialize");
}

Graph CudaDeviceManager::downloadGraph() {
    Graph g(impl->n, impl->m);
    impl->check(pxr_download_graph(impl->need(), g.ranges.data(), g.edges.data()), "downloadGraph");
    return g;
}

std::vector<EdgeIx> CudaDeviceManager::downloadDegrees() {
    std::vector<EdgeIx> d(impl->n);
    impl->check(pxr_download_degrees(impl->need(), d.data()), "downloadDegrees");
    return d;
}

// n entries, the first numActiveNodes of them in sweep order (devSweepCut.h
// downloadPartition copies the whole buffer the same way)
std::vector<NodeData> CudaDeviceManager::downloadPartition() {
    std::vector<NodeData> out(impl->n);
    uint32_t count = 0;
    static_assert(sizeof(NodeData) == sizeof(pxr_node_data), "NodeData layout");
    impl->check(pxr_download_partition(impl->need(), reinterpret_cast<pxr_node_data*>(out.data()), impl->n, &count),
                "downloadPartition");
    return out;
}

void CudaDeviceManager::iterateRandomWalk() { impl->check(pxr_walk_step(impl->need()), "iterateRandomWalk"); }

std::vector<frac_t> CudaDeviceManager::readRandomWalkValues() {
    std::vector<frac_t> x(impl->n);
    impl->check(pxr_read_potentials(impl->need(), x.data()), "readRandomWalkValues");
    return x;
}

void CudaDeviceManager::computeSweepCuts() { impl->check(pxr_sweep(impl->need()), "computeSweepCuts"); }

AllSweepCuts CudaDeviceManager::readSweepCuts() {
    uint32_t count = 0;
    impl->check(pxr_read_sweep_cuts(impl->need(), nullptr, nullptr, 0, &count), "readSweepCuts");
    AllSweepCuts out{std::vector<label_t>(count), std::vector<SweepCutData>(count)};
    static_assert(sizeof(SweepCutData) == sizeof(pxr_sweep_cut), "SweepCutData layout");
    impl->check(pxr_read_sweep_cuts(impl->h, out.clusterIds.data(),
                                    reinterpret_cast<pxr_sweep_cut*>(out.cuts.data()), count, &count),
                "readSweepCuts");
    return out;
}

void CudaDeviceManager::cutClusters() { impl->check(pxr_cut_clusters(impl->need()), "cutClusters"); }

EdgeIx CudaDeviceManager::getNumCutEdges() {
    uint64_t c = 0;
    impl->check(pxr_num_cut_edges(impl->need(), &c), "getNumCutEdges");
    return static_cast<EdgeIx>(c);
}

void CudaDeviceManager::expanderDecomposition() {
    std::printf("Begin Expander Decomposition\n");
    uint32_t rounds = 0;
    const pxr_status s = pxr_decompose(impl->need(), &rounds);
    if (s == PXR_ITER_CAP) std::printf("Not terminating. ABORT.\n");
    else impl->check(s, "expanderDecomposition");
    std::printf("iterations: %u\n", rounds);
}

FinalPartition CudaDeviceManager::getFinalPartition() {
    FinalPartition fp{std::vector<label_t>(impl->n), 0};
    impl->check(pxr_final_partition(impl->need(), fp.clusterIds.data(), &fp.numClusters), "getFinalPartition");
    return fp;
}

std::vector<int> CudaDeviceManager::downloadActiveEdgeMap() {
    std::vector<int> e(2 * static_cast<size_t>(impl->m));
    impl->check(pxr_active_edge_map(impl->need(), e.data()), "downloadActiveEdgeMap");
    return e;
}

std::vector<int> CudaDeviceManager::downloadLabels() {
    std::vector<int> l(impl->n);
    impl->check(pxr_download_labels(impl->need(), l.data()), "downloadLabels");
    return l;
}

// The reference returns 0 here (cuda/device.h:120-123); this returns the
// number of active clusters.
int CudaDeviceManager::getNumClusters() {
    uint32_t k = 0;
    impl->check(pxr_num_active_clusters(impl->need(), &k), "getNumClusters");
    return static_cast<int>(k);
}

// A no-op, as GraphManager::updateLabels is in the reference (cuda/devGraph.h:191-206).
void CudaDeviceManager::updateLabels(std::vector<NodeIx>&, NodeIx) {}
