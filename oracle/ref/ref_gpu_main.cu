// Driver around the reference's own GPU decomposition (test infrastructure).
//
// Compiled by oracle/ref/Makefile from the reference sources where they lie
// (cuda/device.h and the headers it pulls in), with the reference's own CUDA
// flags, into oracle/_ref/ref_gpu.  Nothing here changes the reference code
// path: "decomp" calls CudaDeviceManager::initialize / expanderDecomposition /
// getFinalPartition exactly as main.cpp:42-60 does, and "trace" calls the
// reference's stage functions in the order Impl::expanderDecomposition and
// Impl::cutClusters use (cuda/device.h:101-168, 301-350), copying each
// stage's device state to files in between.  The copies synchronise the
// device but do not alter any value.
//
//   ref_gpu decomp <graph> <seed> <sc> <rw> <outdir>
//   ref_gpu trace  <graph> <seed> <sc> <rw> <rounds_to_dump> <outdir>
//   ref_gpu time   <graph> <seed> <sc> <rw> <repeats>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
#include <thrust/sort.h>
#include <thrust/scan.h>
#include <thrust/reduce.h>
#include <thrust/unique.h>
#include <thrust/binary_search.h>
#include <thrust/random.h>
#include <cub/cub.cuh>
#include <memory>
#include <vector>
#include <string>
#include <iostream>
#include <chrono>
#include <cstdio>

// The trace mode reads the reference's internal device buffers, which are
// private members; open them for this translation unit only.
#define private public
#include "cuda/interface.h"
#include "cuda/device.h"
#undef private

#include "core/partition.h"
#include "pxg_file.h"

// PartitionManager::clusterData has class-default (private) access and no
// getter; name it through an explicit instantiation, which may refer to
// private members.
template <typename Tag, typename Tag::type M>
struct MemberAccess { friend typename Tag::type member_of(Tag) { return M; } };
struct ClusterDataTag {
    typedef thrust::device_vector<ClusterData> PartitionManager::*type;
    friend type member_of(ClusterDataTag);
};
template struct MemberAccess<ClusterDataTag, &PartitionManager::clusterData>;

static Graph load_graph(const std::string& path) {
    PxgFile f = pxg_read(path);
    std::vector<NodeIx> cols(f.cols.begin(), f.cols.end());
    std::vector<EdgeIx> rg(f.offsets.begin(), f.offsets.end());
    return Graph(std::move(cols), std::move(rg), (NodeIx)f.n, (EdgeIx)f.m);
}

template <typename T>
static void dump_dev(const std::string& path, const T* dptr, size_t count) {
    std::vector<T> h(count);
    if (count) cudaMemcpy(h.data(), dptr, count * sizeof(T), cudaMemcpyDeviceToHost);
    raw_write(path, h.data(), count);
}

template <typename T>
static void dump_vec(const std::string& path, thrust::device_vector<T>& v, size_t count) {
    dump_dev(path, thrust::raw_pointer_cast(v.data()), count);
}

static void set_globals(char** argv) {
    randSeed = (unsigned int)std::stoull(argv[3]);
    sc_threshold = std::stof(argv[4]);
    rw_threshold = std::stof(argv[5]);
}

// main.cpp:54-60: the application recounts cut edges on the CPU from the
// final labels with Partition::splitByIndices.
static void cpu_recount(Graph& G, const FinalPartition& fpt, unsigned long long& clusters,
                        unsigned long long& cut) {
    Partition part(&G);
    std::vector<NodeIx> mod;
    part.splitByIndices<false, false>(0, fpt.clusterIds, fpt.numClusters, mod);
    clusters = part.numClusters();
    cut = part.getNumCutEdges();
}

static int run_decomp(char** argv) {
    set_globals(argv);
    std::string out = argv[6];
    Graph G = load_graph(argv[2]);
    Graph Gcopy = G;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    auto t0 = std::chrono::steady_clock::now();
    CudaDeviceManager cuda;
    cuda.initialize(G);
    cudaDeviceSynchronize();
    cudaEventRecord(e0);
    cuda.expanderDecomposition();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    auto t1 = std::chrono::steady_clock::now();
    float loop_ms = 0; cudaEventElapsedTime(&loop_ms, e0, e1);
    FinalPartition fpt = cuda.getFinalPartition();
    EdgeIx devCut = cuda.getNumCutEdges();
    std::vector<int> labels = cuda.downloadLabels();
    unsigned long long clusters = 0, cut = 0;
    cpu_recount(Gcopy, fpt, clusters, cut);
    raw_write(out + "/final_ids.i32", fpt.clusterIds.data(), fpt.clusterIds.size());
    raw_write(out + "/final_labels.i32", labels.data(), labels.size());
    std::printf("{\"mode\": \"decomp\", \"n\": %u, \"m\": %u, \"init_plus_loop_ms\": %.3f, "
                "\"loop_ms\": %.3f, \"num_clusters_fp\": %d, \"clusters_recount\": %llu, "
                "\"cut_edges_recount\": %llu, \"cut_edges_device\": %u}\n",
                G.numNodes, G.numEdges,
                std::chrono::duration<double, std::milli>(t1 - t0).count(), loop_ms,
                fpt.numClusters, clusters, cut, devCut);
    return 0;
}

static int run_time(char** argv) {
    set_globals(argv);
    int reps = std::stoi(argv[6]);
    Graph G = load_graph(argv[2]);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    for (int r = 0; r < reps; ++r) {
        CudaDeviceManager cuda;
        auto t0 = std::chrono::steady_clock::now();
        cuda.initialize(G);
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        cuda.expanderDecomposition();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        FinalPartition fpt = cuda.getFinalPartition();
        auto t1 = std::chrono::steady_clock::now();
        float loop_ms = 0; cudaEventElapsedTime(&loop_ms, e0, e1);
        std::printf("{\"mode\": \"time\", \"rep\": %d, \"m\": %u, \"loop_ms\": %.3f, "
                    "\"e2e_ms\": %.3f, \"num_clusters_fp\": %d}\n",
                    r, G.numEdges, loop_ms,
                    std::chrono::duration<double, std::milli>(t1 - t0).count(), fpt.numClusters);
        std::fflush(stdout);
    }
    return 0;
}

static int run_trace(char** argv) {
    set_globals(argv);
    int dumpRounds = std::stoi(argv[6]);
    std::string out = argv[7];
    Graph G = load_graph(argv[2]);
    Graph Gcopy = G;
    CudaDeviceManager cuda;
    cuda.initialize(G);
    auto& I = *cuda.impl;
    const size_t n = G.numNodes, slots = 2 * (size_t)G.numEdges;

    dump_dev(out + "/x0.f64", I.rw->getValues(), n);
    dump_vec(out + "/deg0.u32", I.pt->getAllInternalDegrees(), n);

    FILE* meta = std::fopen((out + "/meta.jsonl").c_str(), "w");
    int i = 0;
    const int MAX_NUM_ITER = 200000;
    while (i++ < MAX_NUM_ITER && I.pt->numActiveClusters > 0 && I.pt->numActiveNodes > 0) {
        const bool dump = i <= dumpRounds;
        const std::string p = out + "/r" + std::to_string(i) + "_";
        const NodeIx nPre = I.pt->numActiveNodes;
        if (dump) {
            dump_vec(p + "act_pre.ln", I.pt->getActiveNodes(), nPre);
            dump_vec(p + "lab_pre.i32", I.pt->getAllLabels(), n);
            dump_dev(p + "x_pre.f64", I.rw->getValues(), n);
            dump_vec(p + "deg_pre.u32", I.pt->getAllInternalDegrees(), n);
            dump_vec(p + "cols_pre.u32", I.gm->getNeighbors(), slots);
        }
        I.iterateRandomWalk();
        if (dump) {
            dump_dev(p + "x_walk.f64", I.rw->getValues(), n);
            dump_dev(p + "keys.u64", I.sc->getKeyBuffer().Current(), nPre);
        }
        I.computeSweepCuts();
        const NodeIx nPost = I.pt->numActiveNodes;
        const NodeIx kSweep = I.pt->numActiveClusters;
        const NodeIx nCut = I.sc->numClustersWithCut;
        label_t smallest = 0;
        cudaMemcpy(&smallest, I.sc->d_smallestLabel, sizeof(label_t), cudaMemcpyDeviceToHost);
        if (dump) {
            dump_dev(p + "sorted.nd", I.sc->getScNodeData().Current(), nPost);
            dump_vec(p + "act_sorted.ln", I.pt->getActiveNodes(), nPost);
            dump_vec(p + "ulabels.i32", I.pt->getUniqueActiveLabels(), kSweep);
            dump_vec(p + "vols.u32", I.pt->getVolumes(), kSweep);
            dump_vec(p + "allcuts.scd", I.sc->getAllSweepCuts(), kSweep);
            dump_vec(p + "cuts.scd", I.sc->getSweepCuts(), nCut);
        }
        if (nPost == 0) {
            std::fprintf(meta, "{\"round\": %d, \"n_pre\": %u, \"n_post\": 0, \"k_sweep\": %u, "
                         "\"n_cut\": %u, \"smallest\": %d, \"dumped\": %d}\n",
                         i, nPre, kSweep, nCut, smallest, (int)dump);
            break;
        }
        // Impl::cutClusters, one stage at a time (cuda/device.h:163-230).
        if (I.sc->numClustersWithCut > 0)
            I.pt->cutClusters(I.sc->getScNodeData(), I.sc->getSweepCuts(), I.sc->numClustersWithCut);
        if (dump) dump_vec(p + "lab_cut.i32", I.pt->getAllLabels(), n);
        I.cm->consolidate(*I.gm, I.pt->getActiveNodes(), I.pt->getAllLabels(), I.pt->numActiveNodes);
        if (dump) dump_vec(p + "lab_cc.i32", I.pt->getAllLabels(), n);
        I.pt->computeClusterData(I.rw->getValues());
        const NodeIx kData = I.pt->numActiveClusters;
        if (dump) {
            dump_vec(p + "clabels.i32", I.pt->getUniqueActiveLabels(), kData);
            dump_vec(p + "cdata.cd", (*I.pt).*member_of(ClusterDataTag()), kData);
            dump_vec(p + "act_cd.ln", I.pt->getActiveNodes(), nPost);
        }
        I.pt->recenterAndDeactivateClusters(I.rw->getValues(), I.sc->d_smallestLabel);
        const NodeIx kKeep = I.pt->numActiveClusters;
        if (dump) {
            dump_vec(p + "lab_final.i32", I.pt->getAllLabels(), n);
            dump_dev(p + "x_final.f64", I.rw->getValues(), n);
        }
        I.pt->disableEdges(*I.gm);
        if (dump) {
            dump_vec(p + "deg_final.u32", I.pt->getAllInternalDegrees(), n);
            dump_vec(p + "cols_final.u32", I.gm->getNeighbors(), slots);
        }
        std::fprintf(meta, "{\"round\": %d, \"n_pre\": %u, \"n_post\": %u, \"k_sweep\": %u, "
                     "\"n_cut\": %u, \"smallest\": %d, \"k_data\": %u, \"k_keep\": %u, \"dumped\": %d}\n",
                     i, nPre, nPost, kSweep, nCut, smallest, kData, kKeep, (int)dump);
    }
    std::fclose(meta);
    FinalPartition fpt = cuda.getFinalPartition();
    std::vector<int> labels = cuda.downloadLabels();
    raw_write(out + "/final_ids.i32", fpt.clusterIds.data(), fpt.clusterIds.size());
    raw_write(out + "/final_labels.i32", labels.data(), labels.size());
    dump_vec(out + "/final_cols.u32", I.gm->getNeighbors(), slots);
    EdgeIx devCut = cuda.getNumCutEdges();
    unsigned long long clusters = 0, cut = 0;
    cpu_recount(Gcopy, fpt, clusters, cut);
    std::printf("{\"mode\": \"trace\", \"rounds\": %d, \"num_clusters_fp\": %d, \"clusters_recount\": %llu, "
                "\"cut_edges_recount\": %llu, \"cut_edges_device\": %u}\n",
                i, fpt.numClusters, clusters, cut, devCut);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 7 && std::string(argv[1]) == "decomp") return run_decomp(argv);
    if (argc >= 7 && std::string(argv[1]) == "time") return run_time(argv);
    if (argc >= 8 && std::string(argv[1]) == "trace") return run_trace(argv);
    std::fprintf(stderr, "usage: ref_gpu decomp|trace|time <graph> <seed> <sc> <rw> ...\n");
    return 2;
}
