// main.cpp -- the `output` command line, a drop-in for the reference's
// `./output <args>` (src/main.cu:43-407, options src/config.h:14-243).
//
// Same option string "v:f:o:i:k:q:t:d:b:g:n:h", same defaults (hybrid, mvc,
// k=0, q=2^19, t=1.0, d=4, o="1", f="GraphInput.txt"), same input format (a
// header "n m" then m lines "u v" with 1-based ids, src/auxFunctions.cpp:129-209)
// and the same Results/Results.csv row (src/auxFunctions.cpp:580-596).  The
// solve runs through the C ABI (vc_solve); the launch shape is chosen by the
// library, and -q/-t/-d/-b/-g/-n are accepted and recorded in the row as the
// reference does.  Differences, deliberate:
//  * `-v sequential` is refused: this build ships no CPU solver (the reference's
//    CPU path lives only in the test oracle);
//  * the MVC result line reads "Size of minimum vertex cover" (the VC build's
//    wording, main.cu:403) and the row's minimum is the solved size;
//  * the upper-bound heuristics are not run on the host (the device search finds
//    its own incumbent), so maxApprox / edgeApprox are 0 as in the fork's
//    default build (main.cu:76-78);
//  * the graph is checked in O(m log d) (duplicates, self-loops, range,
//    symmetry) instead of the O(V^2) matrix of auxFunctions.cpp:308-354, and a
//    bad file is an error message and exit status 1, not an assert;
//  * Results/ is created when missing.
#include <getopt.h>
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "vcgpu.h"

extern "C" uint32_t vc_debug_stats(int32_t device, int32_t enable, uint64_t *rows, uint32_t max_rows,
                                   uint32_t *launch_shape);

namespace {

enum Version { STACK_ONLY, HYBRID, SEQUENTIAL };
enum Instance { MVC, PVC };

struct Config {
    Version version = HYBRID;
    Instance instance = MVC;
    unsigned k = 0;
    unsigned numBlocks = 0;
    bool userDefMemory = false;
    bool useGlobalMemory = false;
    unsigned blockDim = 0;
    unsigned globalListSize = 1u << 19;
    float globalListThreshold = 1.0f;
    unsigned startingDepth = 4;
    const char *outputFilePrefix = "1";
    const char *graphFileName = "GraphInput.txt";
    bool zeroBased = false;  // -z: vertex ids in the file start at 0
    bool upperBounds = false;  // -u: the reference's two upper-bound heuristics, on the GPU
    bool mcm = false;          // -M: the MCM search of the reference's default (`VC 0`) build
};

void usage()
{
    fprintf(stderr,
            "\nArguments :\n\n"
            "   -v <Version>          hybrid, stackonly, sequential (default hybrid).\n"
            "                         hybrid and stackonly both run the GPU search; sequential\n"
            "                         (the CPU solver) is not part of this build.\n"
            "   -f <Graph File Name>  graph file: \"n m\" then m lines \"u v\", 1-based (default GraphInput.txt)\n"
            "   -o <Output Prefix>    identifier written to Results/Results.csv (default 1)\n"
            "   -i <Instance>         mvc or pvc (default mvc)\n"
            "   -k <parameter>        PVC parameter k (default 0)\n"
            "   -q <Work List Size>   recorded in the results row (default 2^19)\n"
            "   -t <Threshold>        recorded in the results row (default 1.0)\n"
            "   -d <Starting Depth>   recorded in the results row (default 4)\n"
            "   -b <Block Dimension>  recorded; the library picks the launch shape\n"
            "   -g <Use Global Mem>   recorded; the library picks shared or global workspaces\n"
            "   -n <Number of Blocks> recorded; the library sizes the persistent grid\n"
            "   -z                    vertex ids in the graph file start at 0 (the formated_* inputs)\n"
            "   -u                    also run the RemoveMax / RemoveEdge upper-bound heuristics (on the GPU)\n"
            "   -M                    run the MCM search of the reference's default build (VC 0): prints the\n"
            "                         size of maximum matching (mvc, hybrid only; graphs of up to 1024 vertices)\n\n");
}

const char *asString(Version v) { return v == STACK_ONLY ? "stackonly" : (v == HYBRID ? "hybrid" : "sequential"); }
const char *asString(Instance i) { return i == MVC ? "mvc" : "pvc"; }

Config parseArgs(int argc, char **argv)
{
    Config c;
    int opt;
    while ((opt = getopt(argc, argv, "v:f:o:i:k:q:t:d:b:g:n:hzuM")) >= 0) {
        switch (opt) {
        case 'v':
            if (!strcmp(optarg, "stackonly")) c.version = STACK_ONLY;
            else if (!strcmp(optarg, "hybrid")) c.version = HYBRID;
            else if (!strcmp(optarg, "sequential")) c.version = SEQUENTIAL;
            else { fprintf(stderr, "Unrecognized -v option: %s\n", optarg); exit(0); }
            break;
        case 'f': c.graphFileName = optarg; break;
        case 'o': c.outputFilePrefix = optarg; break;
        case 'i':
            if (!strcmp(optarg, "mvc")) c.instance = MVC;
            else if (!strcmp(optarg, "pvc")) c.instance = PVC;
            else { fprintf(stderr, "Unrecognized -i option: %s\n", optarg); exit(0); }
            break;
        case 'k': c.k = (unsigned)atoi(optarg); break;
        case 'q': c.globalListSize = (unsigned)atoi(optarg); break;
        case 't': c.globalListThreshold = (float)atof(optarg); break;
        case 'd': c.startingDepth = (unsigned)atoi(optarg); break;
        case 'b': c.blockDim = (unsigned)atoi(optarg); break;
        case 'g': c.userDefMemory = true; c.useGlobalMemory = atoi(optarg) != 0; break;
        case 'n': c.numBlocks = (unsigned)atoi(optarg); break;
        case 'z': c.zeroBased = true; break;
        case 'u': c.upperBounds = true; break;
        case 'M': c.mcm = true; break;
        case 'h': usage(); exit(0);
        default: fprintf(stderr, "\nUnrecognized option!\n"); exit(0);
        }
    }
    return c;
}

// Reads "n m" and m edges (1-based ids, or 0-based with zero_based) into a
// CSR with sorted rows; false + message on any malformed input.  One pass over
// the file, then a sort of each row, which also finds duplicate edges in
// O(m log d) instead of the reference's O(V^2) check (auxFunctions.cpp:308-354).
bool loadGraph(const char *path, bool zero_based, uint32_t &n, uint32_t &m, std::vector<uint32_t> &rp,
               std::vector<uint32_t> &col, std::string &err)
{
    FILE *f = fopen(path, "rb");
    if (!f) { err = std::string("cannot open ") + path + ": " + strerror(errno); return false; }
    std::vector<char> buf;
    char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    fclose(f);
    buf.push_back('\0');
    char *p = buf.data();
    auto next = [&](unsigned long &out) -> bool {
        while (*p && (*p < '0' || *p > '9')) ++p;
        if (!*p) return false;
        char *e;
        out = strtoul(p, &e, 10);
        p = e;
        return true;
    };
    unsigned long un, um;
    if (!next(un) || !next(um)) { err = "missing \"n m\" header"; return false; }
    n = (uint32_t)un;
    m = (uint32_t)um;
    std::vector<uint32_t> eu(m), ev(m);
    std::vector<uint32_t> deg(n, 0);
    for (uint32_t i = 0; i < m; ++i) {
        unsigned long a, b;
        if (!next(a) || !next(b)) { err = "fewer edges than the header says"; return false; }
        if (!zero_based && (a < 1 || b < 1 || a > n || b > n)) {
            err = "vertex id out of range (ids are 1-based; -z reads 0-based files)";
            return false;
        }
        if (zero_based && (a >= n || b >= n)) { err = "vertex id out of range (ids are 0-based with -z)"; return false; }
        if (a == b) { err = "self-loop"; return false; }
        eu[i] = (uint32_t)(zero_based ? a : a - 1);
        ev[i] = (uint32_t)(zero_based ? b : b - 1);
        ++deg[eu[i]];
        ++deg[ev[i]];
    }
    rp.assign(n + 1, 0);
    for (uint32_t v = 0; v < n; ++v) rp[v + 1] = rp[v] + deg[v];
    col.assign(2ull * m, 0);
    std::vector<uint32_t> pos(rp.begin(), rp.end() - 1);
    for (uint32_t i = 0; i < m; ++i) {
        col[pos[eu[i]]++] = ev[i];
        col[pos[ev[i]]++] = eu[i];
    }
    for (uint32_t v = 0; v < n; ++v) {
        std::sort(col.begin() + rp[v], col.begin() + rp[v + 1]);
        for (uint32_t e = rp[v] + 1; e < rp[v + 1]; ++e)
            if (col[e] == col[e - 1]) { err = "duplicate edge"; return false; }
    }
    return true;
}

struct Bounds {
    unsigned maxApprox = 0, edgeApprox = 0;
    double timeMax = 0, timeEdge = 0;  // seconds
};

void printResults(const Config &c, uint32_t n, uint32_t m, unsigned minimum, unsigned kFound, float ms,
                  const uint32_t *shape, int sms, const Bounds &b)
{
    mkdir("Results", 0755);
    FILE *out = fopen("Results/Results.csv", "a");
    if (!out) { fprintf(stderr, "cannot append to Results/Results.csv\n"); return; }
    const unsigned grid = shape[0], block = shape[1];
    const unsigned per_sm = sms ? grid / (unsigned)sms : 0;
    const int useGlobal = c.userDefMemory ? (int)c.useGlobalMemory : 0;
    fprintf(out, "%s,%s,%u,%u,%s,%s,%d,%f,%d,%d,%d,%u,%d,%d,%u,%f,%u,%f,%u,%u,%u,%f\n", c.outputFilePrefix,
            c.graphFileName, n, m, asString(c.instance), asString(c.version), (int)c.globalListSize,
            c.globalListThreshold, (int)c.startingDepth, useGlobal, (int)block, per_sm, (int)(per_sm * block),
            (int)grid, b.maxApprox, b.timeMax, b.edgeApprox, b.timeEdge, minimum, c.k, kFound, ms);
    fclose(out);
}

// The file's name without its directories (src/Counters.cuh:63-70).
std::string baseName(const char *path)
{
    std::string p(path);
    const size_t k = p.find_last_of('/');
    return k == std::string::npos ? p : p.substr(k + 1);
}

// With VC_COUNTERS=1 in the environment (the reference's USE_COUNTERS build,
// src/Counters.cuh:56-135, main.cu:368-371): NODES_PER_SM/NODES_PER_SM_<prefix>_<file>
// in the reference's layout (a header SM_1..SM_n and one row of tree nodes per
// SM), and Counters/Counters_<prefix>_<file> with one row per search unit.  The
// second file keeps the reference's name and CSV form; its columns are this
// build's counters, because one sweep decides all three reduction rules here
// (phase cycles need a VC_PHASE_TIMERS=1 build, otherwise they read 0).
void printCounters(const Config &c, int sms)
{
    const uint32_t nsu = vc_debug_stats(0, -1, nullptr, 0, nullptr);
    std::vector<uint64_t> rows((size_t)nsu * 16);
    uint32_t shape[5];
    vc_debug_stats(0, -1, rows.data(), nsu, shape);
    const std::string tail = std::string(c.outputFilePrefix) + "_" + baseName(c.graphFileName);
    mkdir("Counters", 0755);
    if (FILE *f = fopen(("Counters/Counters_" + tail).c_str(), "w")) {
        fprintf(f, "SU_NO,NODES,PASSES,DONATIONS,DONATE_FAIL,RECEIVES,ROOTS,BUSY_CYCLES,IDLE_CYCLES,POLLS,RESTORED,"
                   "SMID,SCAN_CYCLES,APPLY_CYCLES,POP_CYCLES,BRANCH_CYCLES\n");
        for (uint32_t i = 0; i < nsu; ++i) {
            fprintf(f, "%u", i);
            for (int j = 0; j < 15; ++j) fprintf(f, ",%llu", (unsigned long long)rows[(size_t)i * 16 + j]);
            fprintf(f, "\n");
        }
        fclose(f);
    }
    std::vector<unsigned long long> per_sm(std::max(sms, 1), 0);
    for (uint32_t i = 0; i < nsu; ++i) {
        const uint64_t sm = rows[(size_t)i * 16 + 10];
        if (sm < per_sm.size()) per_sm[sm] += rows[(size_t)i * 16 + 0];
    }
    mkdir("NODES_PER_SM", 0755);
    if (FILE *f = fopen(("NODES_PER_SM/NODES_PER_SM_" + tail).c_str(), "w")) {
        for (size_t i = 0; i < per_sm.size(); ++i) fprintf(f, "SM_%zu%s", i + 1, i + 1 < per_sm.size() ? "," : "");
        fprintf(f, "\n");
        for (size_t i = 0; i < per_sm.size(); ++i) fprintf(f, "%llu%s", per_sm[i], i + 1 < per_sm.size() ? "," : "");
        fclose(f);
    }
}

}  // namespace

int main(int argc, char **argv)
{
    Config config = parseArgs(argc, argv);
    printf("\nGraph file: %s", config.graphFileName);
    printf("\nUUID: %s\n", config.outputFilePrefix);
    if (config.version == SEQUENTIAL) {
        fprintf(stderr, "-v sequential: the CPU solver is not part of this build; use -v hybrid\n");
        return 1;
    }
    if (config.mcm && (config.version != HYBRID || config.instance != MVC)) {  // main.cu:155-189
        printf("unsupported version %d instance %d\n", (int)config.version, (int)config.instance);
        return 1;
    }
    uint32_t n = 0, m = 0;
    std::vector<uint32_t> rp, col;
    std::string err;
    if (!loadGraph(config.graphFileName, config.zeroBased, n, m, rp, col, err)) {
        fprintf(stderr, "%s: %s\n", config.graphFileName, err.c_str());
        return 1;
    }
    vc_csr g;
    g.n = n;
    g.m = m;
    g.row_ptr = rp.data();
    g.col = col.empty() ? nullptr : col.data();
    g.degree = nullptr;
    Bounds bounds;
    if (config.upperBounds) {  // main.cu:55-74 of the reference, with both heuristics on the GPU
        const uint64_t zero = 0;
        vc_csr_arena a;
        a.count = 1;
        a.n = &n;
        a.row_off = &zero;
        a.col_off = &zero;
        a.row_ptr = rp.data();
        a.col = col.empty() ? nullptr : col.data();
        float ms = 0;
        // rand() right after srand(time(0)), the value the reference's draws use
        srand((unsigned)time(nullptr));
        const uint32_t r = (uint32_t)rand();
        if (vc_remove_max_ub(&a, 0, &bounds.maxApprox, nullptr, &ms) != VC_OK) {
            fprintf(stderr, "GPU Error: RemoveMax upper bound\n");
            return 1;
        }
        bounds.timeMax = ms / 1e3;
        printf("\nElapsed Time for Approximate Remove Max: %f\n", bounds.timeMax);
        printf("Approximate Remove Max Minimum is: %u\n", bounds.maxApprox);
        if (vc_remove_edge_ub(&a, r, 0, &bounds.edgeApprox, nullptr, &ms) != VC_OK) {
            fprintf(stderr, "GPU Error: RemoveEdge upper bound\n");
            return 1;
        }
        bounds.timeEdge = ms / 1e3;
        printf("Elapsed Time for Approximate Remove Edge: %f\n", bounds.timeEdge);
        printf("Approximate Remove Edge Minimum is: %u\n", bounds.edgeApprox);
        fflush(stdout);
    }
    vc_request req;
    memset(&req, 0, sizeof(req));
    req.instance = config.instance == PVC ? VC_PVC : VC_MVC;
    req.k = config.k;
    req.device = 0;
    req.flags = VC_FLAG_NO_VALIDATE;  // loadGraph already checked the file
    std::vector<uint8_t> cover(std::max<uint32_t>(n, 1));
    vc_result res;
    memset(&res, 0, sizeof(res));
    res.cover_mask = cover.data();
    if (config.mcm) {  // main.cu:9-36 (`VC 0`): the maximum starts at 0 (main.cu:240)
        res.cover_mask = nullptr;
        vc_status st = vc_mcm(&g, &req, &res);
        if (st != VC_OK) {
            fprintf(stderr, "GPU Error: %s\n", vc_status_string(st));
            return 1;
        }
        uint32_t shape[5] = {0, 0, 0, 0, 0};
        vc_debug_stats(0, -1, nullptr, 0, shape);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
        printf("\nElapsed time: %fms \n", res.kernel_ms);
        printResults(config, n, m, res.size, 0, res.kernel_ms, shape, sms, bounds);
        printf("\nSize of maximum matching: %u\n\n", res.size / 2);
        return 0;
    }
    const char *counters_env = getenv("VC_COUNTERS");
    const bool counters = counters_env && counters_env[0] == '1';
    if (counters) vc_debug_stats(0, 1, nullptr, 0, nullptr);
    vc_status st = vc_solve(&g, &req, &res);
    if (st != VC_OK) {
        fprintf(stderr, "GPU Error: %s\n", vc_status_string(st));
        return 1;
    }
    uint32_t shape[5] = {0, 0, 0, 0, 0};
    vc_debug_stats(0, -1, nullptr, 0, shape);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    printf("\nOur Config :\n");
    printf("NumOfThreadPerBlocks : %u\n", shape[1]);
    printf("NumOfBlocks : %u\n", shape[0]);
    printf("NumOfSearchUnits : %u\n\n", shape[3]);
    printf("Elapsed time: %fms \n", res.kernel_ms);
    // kFound is the PVC answer; an MVC row keeps it at 0 (main.cu:80, 355-359)
    printResults(config, n, m, res.size, config.instance == PVC ? res.decision : 0, res.kernel_ms, shape, sms, bounds);
    if (counters) printCounters(config, sms);
    if (config.instance == PVC) {
        if (res.decision) printf("\nMinimum is less than or equal to K: %u\n\n", config.k);
        else printf("\nMinimum is greater than K: %u\n\n", config.k);
    } else {
        printf("\nSize of minimum vertex cover: %u\n\n", res.size);
    }
    return 0;
}
