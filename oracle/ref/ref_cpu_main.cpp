// Driver around the reference's own single-threaded CPU code (test infrastructure).
//
// Compiled by oracle/ref/Makefile from the reference's header-only library
// where it lies (lib/core, lib/algorithms), into oracle/_ref/ref_cpu.  Each
// mode calls reference functions unchanged:
//
//   decomp   <graph> <seed> <sc> <rw> <repeats> <out_ids|->
//            expanderDecomposition<Strategy{}>(G, Config{sc, rw}) after
//            random_source.seed(seed) (lib/algorithms/expander_decomposition.h:70-168)
//   walk     <graph> <x_in.f32> <steps> <out.f32>
//            RandomWalk::setData + iterate(part, {0}) (lib/algorithms/random_walk.h:51-70)
//   sweep    <graph> <x_in.f32> <out_prefix>
//            Partition::sweepCut(0, x) (lib/core/partition.h:309-362)
//   cut      <graph> <x_in.f32> <out_ids.i32>
//            sweepCut + split<false,false> as tests/cudaTest.cpp:182-232 does
//   countcut <graph> <ids.i32> <k>
//            Partition::splitByIndices<false,false> as main.cpp:54-60 does
#include "algorithms/expander_decomposition.h"
#include "pxg_file.h"
#include <chrono>
#include <cstdio>

static Graph load_graph(const std::string& path) {
    PxgFile f = pxg_read(path);
    std::vector<NodeIx> cols(f.cols.begin(), f.cols.end());
    std::vector<EdgeIx> rg(f.offsets.begin(), f.offsets.end());
    return Graph(std::move(cols), std::move(rg), (NodeIx)f.n, (EdgeIx)f.m);
}

// Cluster index per vertex, in the partition's cluster order
// (tests/cudaTest.cpp:168-179 builds the same lookup).
static std::vector<int32_t> cluster_ids(const Graph& g, const Partition& part) {
    std::vector<int32_t> ids(g.numNodes, -1);
    int32_t c = 0;
    for (const Cluster& cl : part) {
        for (const ClusterVertex& cv : cl) ids[cv.nix] = c;
        ++c;
    }
    return ids;
}

static int run_decomp(char** argv) {
    const unsigned seed = (unsigned)std::stoul(argv[3]);
    const float sc = std::stof(argv[4]);
    const float rw = std::stof(argv[5]);
    const int reps = std::stoi(argv[6]);
    const std::string out = argv[7];
    for (int r = 0; r < reps; ++r) {
        Graph G = load_graph(argv[2]);
        random_source.seed(seed);
        auto t0 = std::chrono::steady_clock::now();
        Partition part = expanderDecomposition<Strategy{}>(G, Config{sc, rw});
        auto t1 = std::chrono::steady_clock::now();
        part.updateSelfReferences();
        std::printf("{\"mode\": \"decomp\", \"rep\": %d, \"n\": %u, \"m\": %u, \"ms\": %.3f, "
                    "\"clusters\": %u, \"cut_edges\": %u}\n",
                    r, G.numNodes, G.numEdges,
                    std::chrono::duration<double, std::milli>(t1 - t0).count(),
                    part.numClusters(), part.getNumCutEdges());
        std::fflush(stdout);
        if (r == 0 && out != "-") {
            std::vector<int32_t> ids = cluster_ids(G, part);
            raw_write(out, ids.data(), ids.size());
        }
    }
    return 0;
}

static int run_walk(char** argv) {
    Graph G = load_graph(argv[2]);
    std::vector<frac_t> x = raw_read<frac_t>(argv[3], G.numNodes);
    const int steps = std::stoi(argv[4]);
    RandomWalk walk(G.numNodes);
    walk.setData(x);
    Partition part(&G);
    for (int s = 0; s < steps; ++s) walk.iterate(part, {0});
    std::vector<frac_t> y(std::begin(walk.values()), std::end(walk.values()));
    raw_write(argv[5], y.data(), y.size());
    return 0;
}

static int run_sweep(char** argv) {
    Graph G = load_graph(argv[2]);
    std::vector<frac_t> x = raw_read<frac_t>(argv[3], G.numNodes);
    const std::string out = argv[4];
    Partition part(&G);
    SweepCut sc = part.sweepCut(0, x);
    std::vector<uint32_t> order;
    for (const ClusterVertex& cv : part.getCluster(0)) order.push_back(cv.nix);
    std::vector<uint32_t> pre;
    for (const PrefixValues& p : sc.pS) { pre.push_back(p.edgeDiff); pre.push_back(p.vol); }
    raw_write(out + "order.u32", order.data(), order.size());
    raw_write(out + "prefix.u32", pre.data(), pre.size());
    std::printf("{\"mode\": \"sweep\", \"sparsity\": %.9g, \"offset\": %u, \"internal_volume\": %u}\n",
                sc.sparsity, sc.offset, part.getCluster(0).internalVolume);
    return 0;
}

static int run_cut(char** argv) {
    Graph G = load_graph(argv[2]);
    std::vector<frac_t> x = raw_read<frac_t>(argv[3], G.numNodes);
    Partition part(&G);
    SweepCut sc = part.sweepCut(0, x);
    std::vector<NodeIx> modified{0};
    part.split<false, false>(0, sc.offset, modified);
    std::vector<int32_t> ids = cluster_ids(G, part);
    raw_write(argv[4], ids.data(), ids.size());
    std::printf("{\"mode\": \"cut\", \"sparsity\": %.9g, \"offset\": %u, \"clusters\": %u, \"cut_edges\": %u}\n",
                sc.sparsity, sc.offset, part.numClusters(), part.getNumCutEdges());
    return 0;
}

static int run_countcut(char** argv) {
    Graph G = load_graph(argv[2]);
    std::vector<int32_t> ids = raw_read<int32_t>(argv[3], G.numNodes);
    const unsigned k = (unsigned)std::stoul(argv[4]);
    Partition part(&G);
    std::vector<NodeIx> mod;
    part.splitByIndices<false, false>(0, ids, k, mod);
    std::printf("{\"mode\": \"countcut\", \"clusters\": %u, \"cut_edges\": %u}\n",
                part.numClusters(), part.getNumCutEdges());
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string mode = argv[1];
    if (mode == "decomp" && argc >= 8) return run_decomp(argv);
    if (mode == "walk" && argc >= 6) return run_walk(argv);
    if (mode == "sweep" && argc >= 5) return run_sweep(argv);
    if (mode == "cut" && argc >= 5) return run_cut(argv);
    if (mode == "countcut" && argc >= 5) return run_countcut(argv);
    std::fprintf(stderr, "usage: ref_cpu decomp|walk|sweep|cut|countcut ...\n");
    return 2;
}
