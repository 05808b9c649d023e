// Checks the host level layouts (nricp_b200/csrc/host.cpp, build_layout)
// against a direct restatement of what each field must hold, on seeded
// graphs with planted repeated nodes, zero weights and out-of-range nodes.
// Built and run by tests/test_layouts.py; prints "ok" or the first mismatch.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../nricp_b200/csrc/host.hpp"

using namespace nricp_b200;

extern "C" void nricp_default_level(NricpLevelSettings*) {}  // report_json only

namespace {

int failures = 0;

void expect(bool ok, const char* what, int V, int level) {
    if (!ok && failures++ < 10) std::printf("mismatch: %s (V=%d level=%d)\n", what, V, level);
}

void check_level(const TemplateGraph& g, int level, int V) {
    const GraphLevel& G = g.levels[level];
    const LevelLayout L = build_layout(g, level, V);
    const int N = G.node_count();
    const int S = NRICP_MAX_SLOTS;
    // usable slots: in range and weighted, in slot order
    bool usable = L.node_count == N;
    for (int v = 0; v < V && usable; ++v) {
        int c = 0;
        for (int s = 0; s < G.bindings[v].count; ++s) {
            const int n = G.bindings[v].nodes[s];
            if (n < 0 || n >= N || G.bindings[v].weights[s] == 0.0) continue;
            usable &= L.bind_nodes[v * S + c] == n && L.bind_weights[v * S + c] == G.bindings[v].weights[s];
            ++c;
        }
        usable &= L.bind_counts[v] == c;
        for (int s = c; s < S; ++s) usable &= L.bind_nodes[v * S + s] == -1 && L.bind_weights[v * S + s] == 0.0;
    }
    expect(usable, "usable bindings", V, level);
    // gather: each node's (vertex, slot) entries, ascending
    std::vector<int32_t> gather;
    bool gathered = L.gather_begin.size() == static_cast<size_t>(N) + 1 && L.gather_begin[0] == 0;
    for (int n = 0; n < N && gathered; ++n) {
        gather.clear();
        for (int v = 0; v < V; ++v)
            for (int s = 0; s < L.bind_counts[v]; ++s)
                if (L.bind_nodes[v * S + s] == n) gather.push_back(v * S + s);
        gathered &= L.gather_begin[n + 1] - L.gather_begin[n] == static_cast<int32_t>(gather.size()) &&
                    std::equal(gather.begin(), gather.end(), L.gather_entry.begin() + L.gather_begin[n]);
    }
    expect(gathered, "gather lists", V, level);
    // pair groups: every slot pair (x < y) of distinct nodes, in vertex and
    // slot-pair order, stably sorted by (smaller node, larger node)
    struct Entry { int a, b, code; };
    std::vector<Entry> entries;
    for (int v = 0; v < V; ++v)
        for (int x = 0; x < L.bind_counts[v]; ++x)
            for (int y = x + 1; y < L.bind_counts[v]; ++y) {
                const int nx = L.bind_nodes[v * S + x], ny = L.bind_nodes[v * S + y];
                if (nx == ny) continue;
                entries.push_back(nx < ny ? Entry{nx, ny, v * 64 + x * 8 + y} : Entry{ny, nx, v * 64 + y * 8 + x});
            }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const Entry& p, const Entry& q) { return p.a != q.a ? p.a < q.a : p.b < q.b; });
    std::vector<int32_t> nodes, begin, codes;
    for (size_t i = 0; i < entries.size(); ++i) {
        if (i == 0 || entries[i].a != entries[i - 1].a || entries[i].b != entries[i - 1].b) {
            nodes.push_back(entries[i].a);
            nodes.push_back(entries[i].b);
            begin.push_back(static_cast<int32_t>(i));
        }
        codes.push_back(entries[i].code);
    }
    begin.push_back(static_cast<int32_t>(entries.size()));
    expect(L.pair_nodes == nodes && L.pair_begin == begin && L.pair_entry == codes &&
           L.pair_count == static_cast<int>(nodes.size() / 2), "pair groups", V, level);
    // off-diagonal blocks: the pair groups, then each smoothness edge whose
    // node pair shares no vertex, in edge order; an edge whose pair shares one
    // adds into that pair's block
    std::vector<int32_t> blocks = nodes, edge_block;
    for (int e = 0; e < static_cast<int>(G.edges.size() / 2); ++e) {
        const int a = G.edges[e * 2], b = G.edges[e * 2 + 1];
        int found = -1;
        for (int p = 0; p < static_cast<int>(nodes.size() / 2) && found < 0; ++p)
            if (nodes[p * 2] == a && nodes[p * 2 + 1] == b) found = p;
        if (found < 0) {
            found = static_cast<int>(blocks.size() / 2);
            blocks.push_back(a);
            blocks.push_back(b);
        }
        edge_block.push_back(found);
    }
    expect(L.offdiag_nodes == blocks && L.edge_block == edge_block, "off-diagonal blocks", V, level);
    // each block seen from both of its nodes
    const int B = static_cast<int>(blocks.size() / 2);
    bool rows = L.edges == G.edges && static_cast<int>(L.offdiag_nodes.size()) == 2 * B;
    for (int k = 0; k < B && rows; ++k) {
        const int a = L.offdiag_nodes[k * 2], b = L.offdiag_nodes[k * 2 + 1];
        const int ia = L.offdiag_slots[k * 2], ib = L.offdiag_slots[k * 2 + 1];
        rows &= L.row_entry[ia * 2] == k * 2 && L.row_entry[ia * 2 + 1] == b && L.row_entry[ib * 2] == k * 2 + 1 &&
                L.row_entry[ib * 2 + 1] == a && ia >= L.row_begin[a] && ia < L.row_begin[a + 1] &&
                ib >= L.row_begin[b] && ib < L.row_begin[b + 1];
    }
    expect(rows, "off-diagonal rows", V, level);
    // warm start: the reference's four-slot binding to the level before
    bool transfer = true;
    if (level > 0) {
        const std::vector<Binding> tb = bind_vertices(G.rest, g.levels[level - 1].rest, 4, 4);
        for (int n = 0; n < N; ++n) {
            transfer &= L.transfer_counts[n] == tb[n].count;
            for (int s = 0; s < 4; ++s)
                transfer &= L.transfer_nodes[n * 4 + s] == std::max(0, tb[n].nodes[s]) &&
                            L.transfer_weights[n * 4 + s] == tb[n].weights[s];
        }
    }
    expect(transfer, "transfer bindings", V, level);
}

}  // namespace

int main() {
    const int sizes[] = {1, 2, 5, 37, 300, 2562, 9000};
    const int support[] = {1, 2, 4, 8};
    for (int V : sizes)
        for (int k : support) {
            std::mt19937_64 rng(static_cast<uint64_t>(V) * 31 + k);
            std::normal_distribution<double> normal;
            std::vector<double> p(static_cast<size_t>(V) * 3);
            for (double& x : p) x = normal(rng);
            for (int i = 0; i < V / 10; ++i)  // repeated points: distance ties
                for (int c = 0; c < 3; ++c) p[(V - 1 - i) * 3 + c] = p[i * 3 + c];
            TemplateGraph g = build_template_graph(p.data(), V, 3, std::max(1, V / 60), 2, k, 6);
            if (V >= 300) {  // a node in two slots, a zero weight, a node out of range
                Binding& twice = g.levels.back().bindings[7];
                if (twice.count >= 3) twice.nodes[2] = twice.nodes[0];
                Binding& weightless = g.levels.back().bindings[8];
                if (weightless.count >= 2) weightless.weights[1] = 0.0;
                g.levels.back().bindings[9].nodes[0] = 1 << 20;
            }
            for (int l = 0; l < static_cast<int>(g.levels.size()); ++l) check_level(g, l, V);
        }
    std::printf(failures ? "FAILED\n" : "ok\n");
    return failures ? 1 : 0;
}
