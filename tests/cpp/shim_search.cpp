// Uses the reference-shaped C++ interface (include/song_b200.hpp) the way a
// caller of the reference's kernalGraph.h would: KernelGraph, add_vertex via
// the adjacency, upload_to_gpu, gpu_search with a GpuSearchTrace.
// Input file: int32 n, dim, nq, k, ef, block_size, then data[n*dim] f32,
// adj[n*block_size] i32, queries[nq*dim] f32.  Output: ids[nq*k] i32 then
// the traces [nq*12] i32.  With a third argument "extras" it then appends
// Graph::search's results through graph_search (ids [nq*k] i32, -1 padded,
// traces [nq*12] i32) and BitHash(dim, 42, 256).project_all of the queries
// ([nq*8] u32).  Exit 2 with the library's message on failure.
#include <cstdio>
#include <exception>
#include <string>
#include <vector>

#include "song_b200.hpp"

int main(int argc, char** argv) {
    if (argc != 3 && argc != 4) {
        std::fprintf(stderr, "usage: %s input.bin output.bin [extras]\n", argv[0]);
        return 1;
    }
    const bool extras = argc == 4 && std::string(argv[3]) == "extras";
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int h[6];
    if (std::fread(h, 4, 6, f) != 6) return 1;
    const int n = h[0], dim = h[1], nq = h[2], k = h[3], ef = h[4], bs = h[5];
    std::vector<float> data((size_t)n * dim), q((size_t)nq * dim);
    std::vector<int> adj((size_t)n * bs);
    if (std::fread(data.data(), 4, data.size(), f) != data.size() ||
        std::fread(adj.data(), 4, adj.size(), f) != adj.size() ||
        std::fread(q.data(), 4, q.size(), f) != q.size())
        return 1;
    std::fclose(f);
    try {
        song_params p = song_b200::default_params();
        p.block_size = bs;
        p.fixed_degree = bs - 1;
        p.pq_size = 512;
        song_b200::KernelGraph g(n, dim, data, p);
        g.adj = adj;
        g.upload_to_gpu();
        song_b200::GpuSearchTrace trace;
        std::vector<int> ids = song_b200::gpu_search(g, q.data(), nq, k, 512, ef, &trace);
        std::FILE* o = std::fopen(argv[2], "wb");
        std::fwrite(ids.data(), 4, ids.size(), o);
        std::fwrite(trace.queries.data(), sizeof(song_b200::QueryTrace), trace.queries.size(), o);
        if (extras) {
            std::vector<song_b200::QueryTrace> gtr;
            std::vector<std::vector<int>> res = song_b200::graph_search(g, q.data(), nq, k, ef, &gtr);
            for (const auto& r : res) {
                std::vector<int> row(r);
                row.resize((size_t)k, -1);
                std::fwrite(row.data(), 4, row.size(), o);
            }
            std::fwrite(gtr.data(), sizeof(song_b200::QueryTrace), gtr.size(), o);
            song_b200::BitHash bh(dim);
            std::vector<uint32_t> codes = bh.project_all(q.data(), nq);
            std::fwrite(codes.data(), 4, codes.size(), o);
        }
        std::fclose(o);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
    return 0;
}
