// firmcore_baseline: drop-in for the reference CLI (main.cpp:50-451).  Same
// flags (-d -m -o -k -lmd -num_thread -beta), same dataset location
// (../dataset/<d>/ relative to the working directory, main.cpp:98), same
// method names and the same stdout lines, computed on the GPU through
// libfirmcore.  -num_thread is accepted and echoed; it has no effect.
//
// Methods: ParGrid, ParGridPlus, CoreIndex, ParCoreIndex (the core table),
// WdsList, WdsCoreIndex (densest subgraph), fcgrid (kupper/lmdupper report),
// kpe with -k/-lmd (writes one cell to ../output/, FCTree::saveCoreToLocal).
// Extra flag: -table <file> writes the L*n uint32 table (lambda-major).
#include <sys/resource.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "firmcore.h"

using std::cout;
using std::endl;
using std::string;

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// peak resident set size in MB (Util/MemoryUtils.h getPeakRSS / GetPeakRSSInMB)
static long double peak_rss_mb() {
    struct rusage ru;
    getrusage(RUSAGE_SELF, &ru);
    return (long double)ru.ru_maxrss * 1024.0L / (1024.0L * 1024.0L);
}

static int fail(const char* what, fc_status s) {
    std::cerr << "firmcore_baseline: " << what << ": " << fc_status_string(s) << endl;
    return 1;
}

int main(int argc, char* argv[]) {
    string dataset = "example";
    string method = "serial";
    int order = 0;
    unsigned k = 0, lmd = 0, num_thread = 1;
    double beta = 1.0;
    string table_out;
    for (int i = 1; i < argc; i++) {
        string arg = argv[i];
        if (arg == "-d" && i + 1 < argc) dataset = argv[++i];
        if (arg == "-m" && i + 1 < argc) method = argv[++i];
        if (arg == "-o" && i + 1 < argc) order = std::atoi(argv[++i]);
        if (arg == "-k" && i + 1 < argc) k = std::atoi(argv[++i]);
        if (arg == "-lmd" && i + 1 < argc) lmd = std::atoi(argv[++i]);
        if (arg == "-num_thread" && i + 1 < argc) num_thread = std::atoi(argv[++i]);
        if (arg == "-beta" && i + 1 < argc) beta = std::atof(argv[++i]);
        if (arg == "-table" && i + 1 < argc) table_out = argv[++i];
    }
    if (dataset == "") cout << "Use the default dataset example as the user did not specify the dataset" << endl;
    if (method == "") cout << "Use the FirmCore Tree Serial method as the user did not specify the method" << endl;
    cout << "method = " << method << " dataset = " << dataset << endl;

    fc_graph* g = nullptr;
    fc_status s = fc_graph_load_dir(("../dataset/" + dataset + "/").c_str(), order, 1, &g);
    if (s != FC_OK) return fail("loading the dataset", s);
    const uint32_t n = fc_graph_n(g), L = fc_graph_layers(g);
    std::vector<uint32_t> ord(L);
    fc_graph_order(g, ord.data());
    if (order == 1 || order == 2) {
        cout << "Graph order set to: [ ";
        for (uint32_t i = 0; i < L; i++) {
            float density = (float)(fc_graph_layer_m(g, i) >> 1) / (float)n;
            cout << "l" << ord[i] << "(" << density << ") ";
        }
        cout << "]." << endl;
    }
    for (uint32_t i = 0; i < L; i++) cout << ord[i] << " ";
    cout << endl;
    {
        // MultilayerGraph::PrintStatistics (MultilayerGraph.cpp:168-178), uint arithmetic
        unsigned max_m = 0, sum_m = 0;
        for (uint32_t i = 0; i < L; i++) {
            unsigned m = (unsigned)fc_graph_layer_m(g, i) >> 1;
            max_m = std::max(max_m, m);
            sum_m += m;
        }
        cout << "|L| = " << L << ", |V| = " << n << ", |E| = " << sum_m << ", max_|E_i| = " << max_m << endl;
    }

    if (method == "fcgrid") {
        int kupper = 0;
        std::vector<uint64_t> off((uint64_t)L * (n + 1));
        fc_graph_csr(g, off.data(), nullptr);
        for (uint32_t l = 0; l < L; l++)
            for (uint32_t v = 0; v < n; v++) {
                const uint64_t* o = off.data() + (uint64_t)l * (n + 1);
                kupper = std::max(kupper, (int)(o[v + 1] - o[v]));
            }
        method = (L <= (uint32_t)kupper) ? "lmdlist" : "klist";
        cout << "kupper = " << kupper << endl;
        cout << "lmdupper = " << L << endl;
        cout << "method = " << method << endl;
    }

    std::vector<uint32_t> table;
    auto run_table = [&](double& secs) -> fc_status {
        table.assign((size_t)n * L, 0);
        double t0 = now_s();
        fc_status st = fc_coreindex(g, table.data(), 0, nullptr);
        secs = now_s() - t0;
        return st;
    };
    auto write_table = [&]() {
        if (table_out.empty()) return;
        std::ofstream f(table_out, std::ios::binary);
        f.write((const char*)table.data(), (std::streamsize)table.size() * 4);
    };
    double secs = 0;
    if (method == "ParGrid" || method == "ParGridPlus" || method == "CoreIndex" || method == "ParCoreIndex") {
        if (method == "ParGrid") cout << "#thread = " << num_thread << endl;
        if (method == "CoreIndex" || method == "ParCoreIndex") {
            cout << (method == "CoreIndex" ? "I am the CoreIndex" : "I am the ParCoreIndex") << endl;
            cout << "n_layer = " << L << endl;
            cout << "n_vertex = " << n << endl;
        }
        if ((s = run_table(secs)) != FC_OK) return fail(method.c_str(), s);
        if (method == "ParGrid") cout << "Path left Core Parallel Sync Elapsed time: " << secs << " seconds\n";
        if (method == "ParGridPlus") cout << "Mix Core/Path Parallel Sync Elapsed time: " << secs << " seconds\n";
        if (method == "CoreIndex") cout << "CoreIndex Serial Elapsed time: " << secs << " seconds\n";
        if (method == "ParCoreIndex") cout << "CoreIndex Parallel Elapsed time: " << secs << " seconds\n";
        cout << "mem = " << peak_rss_mb() << " MB" << endl;
        write_table();
    }

    if (method == "WdsList" || method == "WdsCoreIndex") {
        if (method == "WdsCoreIndex") {
            cout << "I am the WDS CoreIndex" << endl;
            cout << "n_layer = " << L << endl;
            cout << "n_vertex = " << n << endl;
        }
        fc_densest_result r;
        double t0 = now_s();
        s = fc_densest(g, &beta, 1, &r, nullptr);
        secs = now_s() - t0;
        if (s != FC_OK) return fail(method.c_str(), s);
        cout << "maximum_density = " << r.max_density_f << endl;
        cout << "res_k = " << r.k << endl;
        cout << "res_lmd = " << r.lmd << endl;
        if (method == "WdsList") {
            cout << "res_len = " << r.length << endl;
            cout << "Wds Fctree Elapsed time: " << secs << " seconds\n";
            string resfilename = dataset + "-" + method + "-" + std::to_string(num_thread);
            std::ofstream outfile(resfilename, std::ios::app);
            if (outfile.is_open()) {
                outfile << std::fixed << std::setprecision(6) << "Elapsed time: " << secs << " seconds\n"
                        << "-----------------------------\n";
                outfile.close();
                cout << "Results saved to result.txt\n";
            } else {
                std::cerr << "Error: unable to open result.txt\n";
            }
        } else {
            cout << "Wds CoreIndex Time = " << secs << endl;
        }
    }

    if (method == "kpe") {
        // the kpe run, then one cell written out with original ids
        // (main.cpp:197-225, FCTree::saveCoreToLocal Core/FCTree.cpp:138-153)
        if ((s = run_table(secs)) != FC_OK) return fail(method.c_str(), s);
        cout << "Serial Elapsed time: " << secs << " seconds\n";
        cout << "mem = " << peak_rss_mb() << " MB" << endl;
        if (k != 0 && lmd != 0) {
            cout << k << " " << lmd << endl;
            std::vector<uint32_t> cell;
            if (lmd >= 1 && (uint32_t)lmd <= L) {
                cell.resize(n);
                uint32_t cnt = 0;
                s = fc_cell_members(g, (uint32_t)k, (uint32_t)lmd, cell.data(), n, &cnt, nullptr);
                if (s != FC_OK) return fail(method.c_str(), s);
                cell.resize(cnt);
            }
            if (cell.empty()) {
                cout << "No statisfy result" << endl;
            } else {
                std::vector<uint64_t> id2vtx(n);
                fc_graph_id2vtx(g, id2vtx.data());
                string res_file = "../output/" + dataset + "_k_" + std::to_string(k) + "_lmd_" +
                                  std::to_string(lmd) + "_serial.txt";
                cout << "res_file = " << res_file << endl;
                std::ofstream f(res_file);
                f << "########## k_" + std::to_string(k) + "_lmd_" + std::to_string(lmd) + "_length_" +
                         std::to_string(cell.size())
                  << endl;
                for (uint32_t v : cell) f << id2vtx[v] << endl;
            }
        }
        write_table();
    }
    fc_graph_free(g);
    return 0;
}
