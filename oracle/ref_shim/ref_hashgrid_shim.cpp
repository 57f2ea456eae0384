/*
 * ref_hashgrid_shim.cpp -- C entry points over the reference's own spatial
 * hash grid, physgrad::sparse::SpatialHashGrid<float, uint32_t>
 * (src/sparse_data_structures.h:44-296), compiled as host C++ from its
 * unmodified header by oracle/Makefile into oracle/_ref/libref_hashgrid.so.
 * TEST INFRASTRUCTURE ONLY: pins the oracle's restatement (oracle/hashgrid.py)
 * and generates the golden fixture of tests/golden/.  It only calls the
 * class's public API (constructor, buildHashTable, getNeighbors, accessors).
 */
#include <cstdint>
#include <vector>

#include "sparse_data_structures.h"

using Grid = physgrad::sparse::SpatialHashGrid<float, uint32_t>;

extern "C" {

void* ref_hashgrid_create(float cell_size, const float* dmin, const float* dmax, uint32_t max_particles) {
    return new Grid(cell_size, {dmin[0], dmin[1], dmin[2]}, {dmax[0], dmax[1], dmax[2]}, max_particles);
}

void ref_hashgrid_destroy(void* g) { delete static_cast<Grid*>(g); }

uint32_t ref_hashgrid_total_cells(void* g) { return static_cast<Grid*>(g)->getTotalCells(); }

// buildHashTable over n positions [n][3]; copies the table out (counts and
// starts: total_cells entries; indices: n entries)
void ref_hashgrid_build(void* g, const float* pos, uint32_t n, uint32_t* counts, uint32_t* starts,
                        uint32_t* indices) {
    Grid* G = static_cast<Grid*>(g);
    std::vector<float> p(pos, pos + 3 * (size_t)n);
    G->buildHashTable(p, n);
    const auto& c = G->getCellParticleCounts();
    const auto& s = G->getCellStartIndices();
    const auto& ix = G->getParticleIndices();
    for (size_t i = 0; i < c.size(); ++i) counts[i] = c[i];
    for (size_t i = 0; i < s.size(); ++i) starts[i] = s[i];
    for (uint32_t i = 0; i < n; ++i) indices[i] = ix[i];
}

// getNeighbors of nq queries [nq][3]: offsets [nq + 1]; out receives the
// concatenated lists when cap is large enough.  Returns the total length.
int64_t ref_hashgrid_neighbors(void* g, const float* q, int64_t nq, float radius, int64_t* offsets, uint32_t* out,
                               int64_t cap) {
    Grid* G = static_cast<Grid*>(g);
    int64_t total = 0;
    for (int64_t i = 0; i < nq; ++i) {
        std::vector<uint32_t> nb = G->getNeighbors(q[3 * i], q[3 * i + 1], q[3 * i + 2], radius);
        offsets[i] = total;
        for (uint32_t v : nb) {
            if (total < cap) out[total] = v;
            ++total;
        }
    }
    offsets[nq] = total;
    return total;
}
}
