// Test infrastructure, not product code: the reference checker.
//
// Links the reference's own hot-path objects (compiled in place from the
// reference sources by oracle/Makefile) and drives its public entry points so
// that their results can be read back:
//
//   table   core index table through CoreIndex's get_index2
//           (CoreIndexParallel/CoreIndex.cpp:62-109), one fresh degree table
//           per lambda exactly as CoreIndex::Execute does (:168-213).
//   pgtable the same table through ParGrid's own PeelSync
//           (CoreParallel/FCSyncLeft.cpp:40-131) on ParGrid's schedule
//           (:134-200), snapshotting `valid` after every call.  The stored
//           coreNodeP::valid arrays are not read: PathByK overwrites them in
//           place (:160,167), so node (k,l) ends up holding C_{k+1,l}.
//   wds     FCPathLevelLeft::Execute(mg, tree, true, beta)
//           (Core/FCPathLevelLeft.cpp:311-377) followed by
//           FCTree::WeightDenestSubgraph (Core/FCTree.cpp:69-82) as main.cpp
//           does for `-m WdsList` (main.cpp:402-424); prints the per-cell
//           records of the tree and the winning cell's node set.
//   bench   times the reference's methods on the same loaded graph as
//           main.cpp times them: ParGrid (FCSyncLeft::Execute, main.cpp:
//           229-239), ParGridPlus (FCSyncLeft::ExecuteMix, :277-291),
//           ParCoreIndex (CoreIndex::ExecuteParallel, :378-385) and WdsList
//           (:402-418), W warm-up then K timed runs of the listed ones.
//
// Input is either a dataset directory loaded by the reference's own
// MultilayerGraph::LoadFromFile (Graph/MultilayerGraph.cpp:65-102), or an
// "FCG1" binary edge file (raw (u,v) pairs per layer, in file order).  For a
// binary file the harness applies the loader's id remap itself (first-seen
// order, u before v, self-loops dropped: MultilayerGraph.cpp:122-156) and then
// calls the reference's own Graph::BuildFromEdgeLst (Graph/Graph.cpp:17-50)
// per layer; only the text parse is skipped.
#include "header.h"
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <chrono>
// MultilayerGraph keeps its fields private and has no setter; the binary-input
// path fills them directly.
#define private public
#include "Graph/MultilayerGraph.h"
#undef private
#include "CoreIndexParallel/CoreIndex.h"
#include "CoreParallel/FCCoreTree.h"
#include "CoreParallel/FCSyncLeft.h"
#include "Core/FCTree.h"
#include "Core/FCPathLevelLeft.h"

// External linkage in CoreIndexParallel/CoreIndex.cpp:62.
uint* get_index2(MultilayerGraph &mg, uint **degs, uint lmd, ll_uint *id2vtx);

static void die(const char* m) { fprintf(stderr, "ref_harness: %s\n", m); exit(2); }

static void load_bin(MultilayerGraph& mg, const char* path, std::vector<ll_uint>& id2vtx) {
    FILE* f = fopen(path, "rb");
    if (!f) die("cannot open binary graph");
    char magic[4];
    uint32_t L;
    if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "FCG1", 4) != 0) die("bad magic");
    if (fread(&L, 4, 1, f) != 1) die("short read");
    mg.n_layers = L;
    mg.graph_layers = new Graph[L];
    mg.order = new uint[L];
    for (uint i = 0; i < L; i++) mg.order[i] = i;
    std::unordered_map<ll_uint, uint> vtx2id;
    std::vector<edge*> bufs(L);
    std::vector<uint> sizes(L);
    std::vector<uint32_t> pairs;
    for (uint32_t l = 0; l < L; l++) {
        uint64_t m;
        if (fread(&m, 8, 1, f) != 1) die("short read");
        pairs.resize(2 * m);
        if (m && fread(pairs.data(), 8, m, f) != m) die("short read");
        edge* eb = new edge[2 * m + 2];
        uint ne = 0;
        for (uint64_t i = 0; i < m; i++) {
            uint u = pairs[2 * i], v = pairs[2 * i + 1];
            if (u == v) continue;
            uint uid, vid;
            auto it = vtx2id.find(u);
            if (it != vtx2id.end()) uid = it->second;
            else { uid = (uint)vtx2id.size(); vtx2id.emplace(u, uid); id2vtx.push_back(u); }
            it = vtx2id.find(v);
            if (it != vtx2id.end()) vid = it->second;
            else { vid = (uint)vtx2id.size(); vtx2id.emplace(v, vid); id2vtx.push_back(v); }
            eb[ne++] = edge(uid, vid);
            eb[ne++] = edge(vid, uid);
        }
        bufs[l] = eb;
        sizes[l] = ne;
    }
    fclose(f);
    mg.n = (uint)vtx2id.size();
    for (uint32_t l = 0; l < L; l++) {
        mg.graph_layers[l].BuildFromEdgeLst(bufs[l], mg.n, sizes[l]);
        delete[] bufs[l];
    }
}

static uint** fresh_degs(MultilayerGraph& mg) {
    uint n = mg.GetN(), L = mg.getLayerNumber();
    uint** d = new uint*[n];
    for (uint v = 0; v < n; v++) {
        d[v] = new uint[L];
        for (uint l = 0; l < L; l++) d[v][l] = mg.GetGraph(l).GetAdjLst()[v][0];
    }
    return d;
}
static void free_degs(uint** d, uint n) { for (uint v = 0; v < n; v++) delete[] d[v]; delete[] d; }

static void emit_table(const std::vector<std::vector<uint>>& t, const char* out) {
    FILE* f = fopen(out, "wb");
    if (!f) die("cannot open output");
    for (auto& row : t) fwrite(row.data(), 4, row.size(), f);
    fclose(f);
}

// With threads > 1 the lambda columns run in parallel, each on its own fresh
// degree table, as CoreIndex::ExecuteParallel runs them (CoreIndex.cpp:
// 252-275).
static void mode_table(MultilayerGraph& mg, const char* out, int threads) {
    uint n = mg.GetN(), L = mg.getLayerNumber();
    std::vector<std::vector<uint>> t(L, std::vector<uint>(n));
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (uint lmd = 1; lmd <= L; lmd++) {
        uint** d = fresh_degs(mg);
        uint* c = get_index2(mg, d, lmd, nullptr);
        memcpy(t[lmd - 1].data(), c, 4ull * n);
        delete[] c;
        free_degs(d, n);
    }
    emit_table(t, out);
}

static void free_nodeP(coreNodeP* x, uint n) {
    delete[] x->valid;
    if (x->degs) { for (uint v = 0; v < n; v++) delete[] x->degs[v]; delete[] x->degs; }
    delete x;
}

static void mode_pgtable(MultilayerGraph& mg, const char* out, int threads) {
    omp_set_num_threads(threads);
    uint n = mg.GetN(), L = mg.getLayerNumber();
    std::vector<std::vector<uint>> t(L, std::vector<uint>(n, 0));
    int** degs = new int*[n];
    for (uint v = 0; v < n; v++) {
        degs[v] = new int[L];
        for (uint l = 0; l < L; l++) degs[v][l] = mg.GetGraph(l).GetAdjLst()[v][0];
    }
    bool* valid = new bool[n];
    memset(valid, 1, n);
    int total = 0;
    UtilStats st;
    std::vector<coreNodeP*> spine;
    // lambda spine at k = 1 (PathSerialSync, FCSyncLeft.cpp:134-152)
    for (uint lmd = 1; lmd <= L; lmd++) {
        coreNodeP* node = new coreNodeP();
        FCSyncLeft::PeelSync(mg, degs, 1, lmd, node, valid, true, total, st);
        for (uint v = 0; v < n; v++) if (valid[v]) t[lmd - 1][v] = 1;
        if (total >= (int)n) { delete node; break; }
        spine.push_back(node);
    }
    // k chains per spine node (BuildSubFCTreeSync / PathByK, :155-200), each
    // on a private copy of the spine node's stored arrays.
    for (coreNodeP* s : spine) {
        bool* v2 = new bool[n];
        memcpy(v2, s->valid, n);
        int** d2 = new int*[n];
        for (uint v = 0; v < n; v++) { d2[v] = new int[L]; memcpy(d2[v], s->degs[v], 4ull * L); }
        int tot = s->total;
        for (uint k = 2;; k++) {
            coreNodeP* node = new coreNodeP();
            FCSyncLeft::PeelSync(mg, d2, k, s->lmd, node, v2, false, tot, st);
            bool any = false;
            for (uint v = 0; v < n; v++) if (v2[v]) { t[s->lmd - 1][v] = k; any = true; }
            free_nodeP(node, n);
            if (!any || tot >= (int)n) break;
        }
        delete[] v2;
        for (uint v = 0; v < n; v++) delete[] d2[v];
        delete[] d2;
    }
    for (coreNodeP* s : spine) free_nodeP(s, n);
    for (uint v = 0; v < n; v++) delete[] degs[v];
    delete[] degs;
    delete[] valid;
    emit_table(t, out);
}

static void free_tree(coreNode* x, uint n) {
    if (!x) return;
    free_tree(x->left, n);
    free_tree(x->right, n);
    delete[] x->core;
    delete[] x->o_core;
    delete[] x->o_pos;
    if (x->degs) { for (uint v = 0; v < n; v++) delete[] x->degs[v]; delete[] x->degs; }
    delete x;
}

static void mode_wds(MultilayerGraph& mg, double beta, int threads, const char* out) {
    omp_set_num_threads(threads);
    uint n = mg.GetN();
    uint res_k = 0, res_lmd = 0, res_len = 0;
    float maximum_density = 0.0f;
    FCTree tree(1, 1, n);
    FCPathLevelLeft::Execute(mg, tree, true, beta);
    tree.WeightDenestSubgraph(tree.getNode(), maximum_density, res_k, res_lmd, res_len);
    FILE* f = fopen(out, "w");
    if (!f) die("cannot open output");
    fprintf(f, "result %.9g %u %u %u\n", (double)maximum_density, res_k, res_lmd, res_len);
    // every cell of the tree in WeightDenestSubgraph's preorder
    std::vector<coreNode*> st;
    st.push_back(tree.getNode());
    coreNode* win = nullptr;
    while (!st.empty()) {
        coreNode* x = st.back();
        st.pop_back();
        if (!x || x->k == 0 || x->lmd == 0) continue;
        fprintf(f, "cell %u %u %u %.17g %d\n", x->k, x->lmd, x->length, x->layer_density,
                x->num_select_layer);
        if (x->k == res_k && x->lmd == res_lmd && !win) win = x;
        st.push_back(x->right);
        st.push_back(x->left);
    }
    if (win) {
        std::vector<uint> nodes(win->core, win->core + win->length);
        std::sort(nodes.begin(), nodes.end());
        fprintf(f, "nodes");
        for (uint v : nodes) fprintf(f, " %u", v);
        fprintf(f, "\n");
    }
    fclose(f);
    free_tree(tree.getNode(), n);
}

static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The reference's methods as main.cpp times them, one call each; returns
// seconds.  ParGridPlus turns nested parallelism on as main.cpp:278-281 does
// and off again after, so that it does not carry over to the other methods
// (each of which main.cpp runs in a process of its own).
static double time_method(MultilayerGraph& mg, const std::string& m, int threads, double beta,
                          ll_uint* id2vtx, uint* rk, uint* rl, uint* rlen, float* md) {
    uint n = mg.GetN();
    omp_set_num_threads(threads);
    if (m == "ParGrid") {  // main.cpp:229-239
        double t0 = omp_get_wtime();
        FCCoreTree tree(1, 1, n);
        FCSyncLeft::Execute(mg, tree);
        return omp_get_wtime() - t0;
    }
    if (m == "ParGridPlus") {  // main.cpp:277-291
        omp_set_nested(1);
        omp_set_max_active_levels(2);
        omp_set_num_threads(threads);
        double t0 = omp_get_wtime();
        FCCoreTree tree(1, 1, n);
        FCSyncLeft::ExecuteMix(mg, tree);
        double t = omp_get_wtime() - t0;
        omp_set_nested(0);
        omp_set_max_active_levels(1);
        return t;
    }
    if (m == "ParCoreIndex") {  // main.cpp:378-385
        double t0 = omp_get_wtime();
        CoreIndex::ExecuteParallel(mg, id2vtx);
        return omp_get_wtime() - t0;
    }
    if (m == "WdsList") {  // main.cpp:402-418
        double t0 = omp_get_wtime();
        FCTree wt(1, 1, n);
        FCPathLevelLeft::Execute(mg, wt, true, beta);
        double t = omp_get_wtime() - t0;
        wt.WeightDenestSubgraph(wt.getNode(), *md, *rk, *rl, *rlen);
        free_tree(wt.getNode(), n);
        return t;
    }
    die("unknown method");
    return 0;
}

// `methods` is a comma-separated list of ParGrid, ParGridPlus, ParCoreIndex,
// WdsList; every step times each of them once, in that order, and prints one
// STEP line with their seconds.
static void mode_bench(MultilayerGraph& mg, int steps, int warmup, double beta, int threads,
                       const std::string& methods, ll_uint* id2vtx) {
    std::vector<std::string> ms;
    for (size_t a = 0; a <= methods.size();) {
        size_t b = methods.find(',', a);
        if (b == std::string::npos) b = methods.size();
        if (b > a) ms.push_back(methods.substr(a, b - a));
        a = b + 1;
    }
    for (int it = 0; it < warmup + steps; it++) {
        uint rk = 0, rl = 0, rlen = 0;
        float md = 0.0f;
        std::string times;
        for (const std::string& m : ms) {
            double t = time_method(mg, m, threads, beta, id2vtx, &rk, &rl, &rlen, &md);
            char b[96];
            snprintf(b, sizeof(b), ", \"%s\": %.6f", m.c_str(), t);
            times += b;
        }
        printf("STEP {\"step\": %d, \"warmup\": %s%s, \"density\": %.9g, \"k\": %u, "
               "\"lmd\": %u, \"len\": %u}\n",
               it, it < warmup ? "true" : "false", times.c_str(), (double)md, rk, rl, rlen);
        fflush(stdout);
    }
}

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr,
                "usage: ref_harness <dir/|file.fcg> table <out.bin> [threads]\n"
                "       ref_harness <dir/|file.fcg> pgtable <out.bin> [threads]\n"
                "       ref_harness <dir/|file.fcg> wds <out.txt> <beta> [threads]\n"
                "       ref_harness <dir/|file.fcg> bench <steps> <warmup> <beta> <threads> "
                "[methods, default ParGrid,WdsList]\n");
        return 2;
    }
    std::string in = argv[1];
    std::string mode = argv[2];
    MultilayerGraph mg;
    std::vector<ll_uint> id2vtx;
    double tl0 = now();
    if (!in.empty() && in.back() == '/') {
        mg.LoadFromFile(in);
    } else {
        load_bin(mg, in.c_str(), id2vtx);
    }
    double tl1 = now();
    fprintf(stderr, "loaded n=%u L=%u in %.2fs\n", mg.GetN(), mg.getLayerNumber(), tl1 - tl0);
    if (mode == "table") mode_table(mg, argv[3], argc > 4 ? atoi(argv[4]) : 1);
    else if (mode == "pgtable") mode_pgtable(mg, argv[3], argc > 4 ? atoi(argv[4]) : 1);
    else if (mode == "wds") {
        if (argc < 5) die("wds needs beta");
        mode_wds(mg, atof(argv[4]), argc > 5 ? atoi(argv[5]) : 1, argv[3]);
    } else if (mode == "bench") {
        if (argc < 7) die("bench needs steps warmup beta threads");
        if (id2vtx.empty()) {
            id2vtx.resize(mg.GetN());
            mg.LoadId2VtxMap(id2vtx.data());
        }
        mode_bench(mg, atoi(argv[3]), atoi(argv[4]), atof(argv[5]), atoi(argv[6]),
                   argc > 7 ? argv[7] : "ParGrid,WdsList", id2vtx.data());
    } else die("unknown mode");
    return 0;
}
