// ref_bench.cpp -- BENCH / TEST INFRASTRUCTURE ONLY.
//
// Times the reference's own CPU solver on a file of graphs: for MVC its
// RemoveMaxApproximateMVC upper bound (src/auxFunctions.cpp:211) followed by
// Sequential(graph, ub) (src/Sequential.cpp:3); for PVC
// SequentialParameterized(graph, k+1, k) (src/SequentialParameterized.cpp:4).
// The reference solver has no node budget, so every instance runs in its own
// forked child with a wall-time limit; up to `threads` children run at once.
//
//   ref_bench <graphs.bin> <threads> <timeout_s> [total_s]
// With total_s, no new graph starts after total_s seconds; graphs still running
// then are stopped and reported as "cut".
//   graphs.bin: u32 count, then per graph: u32 n, u32 nnz, u32 mode (0 mvc,
//               1 pvc), u32 k, u32 row_ptr[n+1], u32 col[nnz]
// Prints one line per graph: "<index> <ok|timeout|error> <size-or-kFound> <ms>".
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <sys/wait.h>
#include <unistd.h>
#include <vector>

#include "CSRGraphRep.h"
#include "Sequential.h"
#include "SequentialParameterized.h"
#include "auxFunctions.h"

struct G {
    uint32_t n, nnz, mode, k;
    std::vector<uint32_t> rp, col;
};

static double now_ms()
{
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec / 1e6;
}

static CSRGraph make_graph(const G &g)
{
    CSRGraph c;
    c.vertexNum = g.n;
    c.edgeNum = g.nnz / 2;
    c.srcPtr = (unsigned int *)malloc(sizeof(unsigned int) * (g.n + 1));
    c.dst = (unsigned int *)malloc(sizeof(unsigned int) * (g.nnz ? g.nnz : 1));
    c.degree = (int *)malloc(sizeof(int) * (g.n ? g.n : 1));
    c.srcPtrUncompressed = nullptr;
    memcpy(c.srcPtr, g.rp.data(), sizeof(unsigned int) * (g.n + 1));
    if (g.nnz) memcpy(c.dst, g.col.data(), sizeof(unsigned int) * g.nnz);
    for (uint32_t v = 0; v < g.n; ++v) c.degree[v] = (int)(g.rp[v + 1] - g.rp[v]);
    return c;
}

static uint32_t solve(const G &g)
{
    if (g.mode == 1) {
        unsigned int found = 0;
        SequentialParameterized(make_graph(g), g.k + 1, g.k, &found);
        return found;
    }
    CSRGraph c = make_graph(g);
    unsigned int ub = RemoveMaxApproximateMVC(c);
    c.del();
    return Sequential(make_graph(g), ub);
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s graphs.bin threads timeout_s\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    uint32_t count = 0;
    if (fread(&count, 4, 1, f) != 1) return 2;
    std::vector<G> gs(count);
    for (auto &g : gs) {
        uint32_t h[4];
        if (fread(h, 4, 4, f) != 4) return 2;
        g.n = h[0]; g.nnz = h[1]; g.mode = h[2]; g.k = h[3];
        g.rp.resize(g.n + 1);
        g.col.resize(g.nnz);
        if (fread(g.rp.data(), 4, g.n + 1, f) != g.n + 1) return 2;
        if (g.nnz && fread(g.col.data(), 4, g.nnz, f) != g.nnz) return 2;
    }
    fclose(f);
    const int threads = atoi(argv[2]);
    const double timeout_ms = atof(argv[3]) * 1e3;
    const double total_ms = argc > 4 ? atof(argv[4]) * 1e3 : 1e300;
    const double start = now_ms();
    struct Child { pid_t pid; int fd; uint32_t idx; double t0; };
    std::vector<Child> running;
    uint32_t next = 0;
    while ((next < count && now_ms() - start <= total_ms) || !running.empty()) {
        const bool over = now_ms() - start > total_ms;
        while (!over && (int)running.size() < threads && next < count) {
            int p[2];
            if (pipe(p) != 0) return 3;
            double t0 = now_ms();
            pid_t pid = fork();
            if (pid == 0) {
                close(p[0]);
                uint32_t r = solve(gs[next]);
                if (write(p[1], &r, 4) != 4) _exit(1);
                _exit(0);
            }
            close(p[1]);
            running.push_back({pid, p[0], next, t0});
            ++next;
        }
        usleep(200);
        for (size_t i = 0; i < running.size();) {
            Child &c = running[i];
            int st = 0;
            pid_t w = waitpid(c.pid, &st, WNOHANG);
            double el = now_ms() - c.t0;
            if (w == c.pid) {
                uint32_t r = 0;
                bool ok = WIFEXITED(st) && WEXITSTATUS(st) == 0 && read(c.fd, &r, 4) == 4;
                printf("%u %s %u %.3f\n", c.idx, ok ? "ok" : "error", r, el);
                close(c.fd);
                running.erase(running.begin() + i);
            } else if (el > timeout_ms || over) {
                kill(c.pid, SIGKILL);
                waitpid(c.pid, &st, 0);
                printf("%u %s 0 %.3f\n", c.idx, over ? "cut" : "timeout", el);
                close(c.fd);
                running.erase(running.begin() + i);
            } else {
                ++i;
            }
        }
        fflush(stdout);
    }
    return 0;
}
