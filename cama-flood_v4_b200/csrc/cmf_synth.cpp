// cmf_synth.cpp -- native loops of the seeded synthetic-case generator (cmf_b200.synth).
//
// The network generator grows a D8 forest from the river mouths by a randomised priority-first
// search and then walks it twice (upstream-area accumulation, elevation from the outlets).  These
// are sequential loops over every land cell; in Python they dominate the generation of the
// multi-million-cell networks.  Each function performs exactly the operations of the Python
// statement of the same loop (same pop order, same cost sequence, same floating-point operations,
// compiled without contraction), so both give identical cases; the test suite checks that.
#include <cstdint>
#include <queue>
#include <vector>

namespace {

struct Entry {
    double pr;        // accumulated cost
    int64_t cell;     // cell to visit
    int64_t from;     // cell that pushed it (-1 for a mouth)
};

// min-heap on (pr, cell, from): the order in which a heap of those tuples pops them
struct Later {
    bool operator()(const Entry &a, const Entry &b) const {
        if (a.pr != b.pr) return a.pr > b.pr;
        if (a.cell != b.cell) return a.cell > b.cell;
        return a.from > b.from;
    }
};

// (dx, dy) of the 8 neighbours, in the generator's order
const int kNb[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};

}  // namespace

extern "C" {

// Grows the forest over land[ny*nx] (row-major, IX fastest) from the given mouths.  Every popped
// cell pushes each unvisited land neighbour with cost pr + costs[ci] (x 1.4142 on diagonals),
// ci advancing by one per push and wrapping at ncosts.  Outputs down[ncell] (downstream flat index,
// -1 for mouths, -2 for cells never reached) and order[] (cells in visiting order, parents first);
// returns the number of visited cells, or -1 on bad arguments.
int64_t cmf_synth_grow_forest(int32_t nx, int32_t ny, const uint8_t *land, const int64_t *mouths, int64_t nmouths,
                              const double *costs, int64_t ncosts, int64_t *down, int64_t *order) {
    if (nx <= 0 || ny <= 0 || !land || (nmouths > 0 && !mouths) || !costs || ncosts <= 0 || !down || !order) return -1;
    const int64_t ncell = (int64_t)nx * ny;
    std::vector<uint8_t> visited((size_t)ncell, 0);
    for (int64_t c = 0; c < ncell; c++) down[c] = -2;
    std::priority_queue<Entry, std::vector<Entry>, Later> heap;
    for (int64_t k = 0; k < nmouths; k++) {
        if (mouths[k] < 0 || mouths[k] >= ncell) return -1;
        heap.push({0.0, mouths[k], -1});
    }
    int64_t ci = 0, n = 0;
    while (!heap.empty()) {
        const Entry e = heap.top();
        heap.pop();
        const int64_t c = e.cell;
        if (visited[c]) continue;
        visited[c] = 1;
        down[c] = e.from;
        order[n++] = c;
        const int64_t cy = c / nx, cx = c % nx;
        for (const auto &d : kNb) {
            const int64_t jx = cx + d[0], jy = cy + d[1];
            if (jx < 0 || jx >= nx || jy < 0 || jy >= ny) continue;
            const int64_t j = jy * nx + jx;
            if (visited[j] || !land[j]) continue;
            const double w = costs[ci] * ((d[0] && d[1]) ? 1.4142 : 1.0);
            if (++ci >= ncosts) ci = 0;
            heap.push({e.pr + w, j, c});
        }
    }
    return n;
}

// Upstream accumulation in reverse visiting order: upa[down[c]] += upa[c] for every non-mouth c.
void cmf_synth_accumulate(int64_t n, const int64_t *order, const int64_t *down, double *upa) {
    for (int64_t k = n - 1; k >= 0; k--) {
        const int64_t c = order[k], d = down[c];
        if (d >= 0) upa[d] += upa[c];
    }
}

// Elevation from the outlets upward in visiting order: elev[c] = elev[down[c]] + slope[c] * len[c].
void cmf_synth_elevation(int64_t n, const int64_t *order, const int64_t *down, const double *slope, const double *len,
                         double *elev) {
    for (int64_t k = 0; k < n; k++) {
        const int64_t c = order[k], d = down[c];
        if (d >= 0) {
            const double rise = slope[c] * len[c];
            elev[c] = elev[d] + rise;
        }
    }
}

}  // extern "C"
