// firmcore_baseline: drop-in for the reference CLI (main.cpp:50-451).  Same
// flags (-d -m -o -k -lmd -num_thread -beta), same dataset location
// (../dataset/<d>/ relative to the working directory, main.cpp:98), same
// method names and the same stdout lines, computed on the GPU through
// libfirmcore.  -num_thread is accepted and echoed; it has no effect.
//
// Methods: ParGrid, ParGridPlus, CoreIndex, ParCoreIndex (the core table),
// WdsList, WdsCoreIndex (densest subgraph), fcgrid (kupper/lmdupper report),
// kpe with -k/-lmd (writes one cell to ../output/, FCTree::saveCoreToLocal),
// CoreMem / PathMem (every cell in compact form: the cell index),
// CoreIndexTimeOnline / CoreIndexTimeOffline (a list of cells answered from
// the table by a scan / from the cell index) and MLCDTime (the MLCD
// membership test on a coreness file), main.cpp:331-362, 453-582.
// Extra flags:
//   -table <file>  writes the L*n uint32 table (lambda-major);
//   -klmd <file>   the cell list of the query methods, "k lmd" per line
//                  (default ../klmd/<d>_klmd.txt, the reference's klmd/
//                  directory; the reference reads a fixed absolute path);
//   -cores <file>  MLCDTime's coreness file, one node per line, P values each
//                  (default ../cores/<d>_cores.txt);
//   -qout <file>   the query methods write their answers there, one block per
//                  query: "########## k_<k>_lmd_<lmd>_length_<len>", then the
//                  nodes (original ids; MLCDTime: row numbers), one per line;
//   -cells <file>  CoreMem / PathMem write the cell index there (binary,
//                  little-endian: u32 L, u32 n, u64 col_off[L+1],
//                  u32 sizes[col_off[L]], u32 order[L*n]; fc_cell_index).
#include <sys/resource.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
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
    string table_out, klmd_path, cores_path, qout_path, cells_path;
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
        if (arg == "-klmd" && i + 1 < argc) klmd_path = argv[++i];
        if (arg == "-cores" && i + 1 < argc) cores_path = argv[++i];
        if (arg == "-qout" && i + 1 < argc) qout_path = argv[++i];
        if (arg == "-cells" && i + 1 < argc) cells_path = argv[++i];
    }
    if (klmd_path.empty()) klmd_path = "../klmd/" + dataset + "_klmd.txt";
    if (cores_path.empty()) cores_path = "../cores/" + dataset + "_cores.txt";
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
    if (method == "CoreMem" || method == "PathMem") {
        // the table and every cell in compact form (the per-cell difference
        // lists of FCSyncMem / FCPathMem are the blocks of the cell index)
        double t0 = now_s();
        table.assign((size_t)n * L, 0);
        if ((s = fc_coreindex(g, table.data(), 0, nullptr)) != FC_OK) return fail(method.c_str(), s);
        std::vector<uint64_t> col_off(L + 1);
        uint64_t nsizes = 0;
        if ((s = fc_cell_index(g, nullptr, col_off.data(), nullptr, 0, &nsizes, nullptr)) != FC_OK)
            return fail(method.c_str(), s);
        std::vector<uint32_t> sizes(nsizes), order((size_t)n * L);
        if ((s = fc_cell_index(g, order.data(), col_off.data(), sizes.data(), nsizes, &nsizes,
                               nullptr)) != FC_OK)
            return fail(method.c_str(), s);
        secs = now_s() - t0;
        if (method == "CoreMem") {
            cout << "CoreParallel Sync with Memory reduction Elapsed time: " << secs << " seconds\n";
            cout << "CoreParallel Sync with Memory reduction mem = " << peak_rss_mb() << " MB" << endl;
        } else {
            cout << "PathParallel with Memory reduction Elapsed time: " << secs << " seconds\n";
            cout << "PathParallel Sync with Memory reduction mem = " << peak_rss_mb() << " MB" << endl;
        }
        if (!cells_path.empty()) {
            std::ofstream f(cells_path, std::ios::binary);
            f.write((const char*)&L, 4);
            f.write((const char*)&n, 4);
            f.write((const char*)col_off.data(), (std::streamsize)col_off.size() * 8);
            f.write((const char*)sizes.data(), (std::streamsize)sizes.size() * 4);
            f.write((const char*)order.data(), (std::streamsize)order.size() * 4);
        }
        write_table();
    }

    if (method == "CoreIndexTimeOnline" || method == "CoreIndexTimeOffline" || method == "MLCDTime") {
        // the cell list, "k lmd" pairs (main.cpp:458-463, 497-502, 535-540)
        std::vector<uint32_t> ks, lmds;
        {
            std::ifstream in(klmd_path);
            if (!in) return fail(("reading " + klmd_path).c_str(), FC_ERR_IO);
            long long kk, ll;
            while (in >> kk >> ll) {
                // the table methods index klmd[lmd] (size L+1): other lambdas
                // are outside the reference's arrays and are left out here
                if (method != "MLCDTime" && (ll < 1 || ll > (long long)L)) continue;
                ks.push_back((uint32_t)kk);
                lmds.push_back((uint32_t)ll);
            }
        }
        const uint32_t nq = (uint32_t)ks.size();
        std::vector<uint64_t> qoff(nq + 1, 0);
        std::vector<uint32_t> qnodes;
        std::vector<uint64_t> id2vtx;
        if (method == "MLCDTime") {
            // one node per line, its values (main.cpp:466-482); every line
            // must hold as many values as the first
            std::vector<uint32_t> cores;
            uint32_t P = 0, rows = 0;
            std::ifstream in(cores_path);
            if (!in) return fail(("reading " + cores_path).c_str(), FC_ERR_IO);
            string line;
            while (std::getline(in, line)) {
                std::istringstream ls(line);
                long long x;
                uint32_t c = 0;
                while (ls >> x) {
                    cores.push_back((uint32_t)x);
                    c++;
                }
                if (rows == 0) P = c;
                if (c != P) return fail(("ragged row in " + cores_path).c_str(), FC_ERR_PARSE);
                rows++;
            }
            double t0 = now_s();
            s = fc_mlcd_query(cores.data(), rows, P, ks.data(), lmds.data(), nq, qoff.data(), nullptr,
                              0, nullptr);
            if (s == FC_OK) {
                qnodes.resize(qoff[nq]);
                s = fc_mlcd_query(cores.data(), rows, P, ks.data(), lmds.data(), nq, qoff.data(),
                                  qnodes.data(), qnodes.size(), nullptr);
            }
            secs = now_s() - t0;
            if (s != FC_OK) return fail(method.c_str(), s);
        } else {
            // the table first, untimed: the reference reads it from a file
            // (main.cpp:508-519, 546-557) before its timer starts
            if ((s = fc_coreindex(g, nullptr, 0, nullptr)) != FC_OK) return fail(method.c_str(), s);
            const int by_index = method == "CoreIndexTimeOffline";
            double t0 = now_s();
            s = fc_cells_members(g, ks.data(), lmds.data(), nq, by_index, qoff.data(), nullptr, 0,
                                 nullptr);
            if (s == FC_OK) {
                qnodes.resize(qoff[nq]);
                s = fc_cells_members(g, ks.data(), lmds.data(), nq, by_index, qoff.data(),
                                     qnodes.data(), qnodes.size(), nullptr);
            }
            secs = now_s() - t0;
            if (s != FC_OK) return fail(method.c_str(), s);
            id2vtx.resize(n);
            fc_graph_id2vtx(g, id2vtx.data());
        }
        std::cout << "Elapsed time: " << secs << " seconds\n";
        if (!qout_path.empty()) {
            std::ofstream f(qout_path);
            for (uint32_t q = 0; q < nq; q++) {
                f << "########## k_" << ks[q] << "_lmd_" << lmds[q] << "_length_" << qoff[q + 1] - qoff[q]
                  << "\n";
                for (uint64_t i = qoff[q]; i < qoff[q + 1]; i++)
                    f << (id2vtx.empty() ? (uint64_t)qnodes[i] : id2vtx[qnodes[i]]) << "\n";
            }
        }
    }
    fc_graph_free(g);
    return 0;
}
