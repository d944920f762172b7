/* CPU oracle: topology, samplers, kernels and the HNS_Advance step, restated in plain C.
 * TEST INFRASTRUCTURE ONLY -- see hns_oracle.h for what pins it. */
#include "hns_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- topology --------------------------------------------------------------------------
 * Leaf-dense layout of the reference's IndexGridBuilder (src/Utils/GridBuilder.hpp:164-174,
 * 231-251): leaf i owns slots [512 i, 512 i + 512), slot 512 i + n holds the voxel at
 * origin + ((n>>6)&7, (n>>3)&7, n&7) (NanoVDB LeafNode::CoordToOffset,
 * externals/nanovdb/NanoVDB.h:4598-4601). A ValueOnIndex grid over these voxels gives
 * every voxel the offset 1 + slot and 0 to everything outside
 * (LeafData<ValueOnIndex>::getValue, NanoVDB.h:4219-4227) when the leaves are in NanoVDB
 * order. Leaf lookup here is an open-addressing hash over leaf coordinates. */
struct hnso_topo {
    int64_t num_leaves;
    int32_t* origins; /* 3 per leaf */
    uint64_t mask;    /* hash capacity - 1 */
    int64_t* table;   /* leaf index or -1 */
};

static uint64_t hash3(int32_t a, int32_t b, int32_t c) {
    uint64_t h = (uint64_t)(uint32_t)a * 0x9E3779B97F4A7C15ull;
    h ^= (uint64_t)(uint32_t)b * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
    h ^= (uint64_t)(uint32_t)c * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
    return h ^ (h >> 29);
}

hnso_topo* hnso_topo_create(const int32_t* leaf_origins, int64_t num_leaves) {
    hnso_topo* t = (hnso_topo*)calloc(1, sizeof(hnso_topo));
    t->num_leaves = num_leaves;
    t->origins = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(num_leaves > 0 ? num_leaves : 1));
    memcpy(t->origins, leaf_origins, sizeof(int32_t) * 3 * (size_t)num_leaves);
    uint64_t cap = 16;
    while (cap < (uint64_t)(2 * num_leaves)) cap <<= 1;
    t->mask = cap - 1;
    t->table = (int64_t*)malloc(sizeof(int64_t) * cap);
    for (uint64_t q = 0; q < cap; ++q) t->table[q] = -1;
    for (int64_t l = 0; l < num_leaves; ++l) {
        const int32_t* o = t->origins + 3 * l;
        uint64_t h = hash3(o[0] >> 3, o[1] >> 3, o[2] >> 3) & t->mask;
        while (t->table[h] >= 0) h = (h + 1) & t->mask;
        t->table[h] = l;
    }
    return t;
}

void hnso_topo_destroy(hnso_topo* t) {
    if (!t) return;
    free(t->origins);
    free(t->table);
    free(t);
}

int64_t hnso_topo_num_voxels(const hnso_topo* t) { return t->num_leaves * 512; }

static inline const int32_t* hnso_leaf_origin(const hnso_topo* t, int64_t leaf) { return t->origins + 3 * leaf; }

static inline int64_t find_leaf(const hnso_topo* t, int32_t i, int32_t j, int32_t k) {
    const int32_t a = i >> 3, b = j >> 3, c = k >> 3;
    uint64_t h = hash3(a, b, c) & t->mask;
    for (;;) {
        const int64_t l = t->table[h];
        if (l < 0) return -1;
        const int32_t* o = t->origins + 3 * l;
        if ((o[0] >> 3) == a && (o[1] >> 3) == b && (o[2] >> 3) == c) return l;
        h = (h + 1) & t->mask;
    }
}

uint64_t hnso_offset(const hnso_topo* t, int32_t i, int32_t j, int32_t k) {
    const int64_t l = find_leaf(t, i, j, k);
    if (l < 0) return 0;
    return 1u + (uint64_t)l * 512u + (uint64_t)(((i & 7) << 6) | ((j & 7) << 3) | (k & 7));
}

void hnso_offsets(const hnso_topo* t, const int32_t* ijk, int64_t n, uint64_t* out) {
    for (int64_t q = 0; q < n; ++q) out[q] = hnso_offset(t, ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]);
}

void hnso_slot_coords(const hnso_topo* t, int32_t* out) {
    for (int64_t l = 0; l < t->num_leaves; ++l) {
        const int32_t* o = t->origins + 3 * l;
        for (int n = 0; n < 512; ++n) {
            int32_t* c = out + 3 * (l * 512 + n);
            c[0] = o[0] + ((n >> 6) & 7);
            c[1] = o[1] + ((n >> 3) & 7);
            c[2] = o[2] + (n & 7);
        }
    }
}

/* NanoVDB leaf order: root tiles (4096^3) in signed (x, y, z) order, then upper-node child
 * index (32^3 children of 128^3), then lower-node child index (16^3 leaves). This is the
 * order of the device builder's radix sorts (externals/nanovdb/tools/cuda/PointsToGrid.cuh:
 * 596-651: biased 21-bit tile keys, then upper/lower/voxel offsets) and of the host
 * builder's std::map root (tools/GridBuilder.h:65). */
static int cmp_leaf(const void* pa, const void* pb) {
    const int32_t* a = (const int32_t*)pa;
    const int32_t* b = (const int32_t*)pb;
    for (int d = 0; d < 3; ++d) {
        const int32_t x = a[d] >> 12, y = b[d] >> 12;
        if (x != y) return x < y ? -1 : 1;
    }
    for (int d = 0; d < 3; ++d) {
        const int32_t x = (a[d] >> 7) & 31, y = (b[d] >> 7) & 31;
        if (x != y) return x < y ? -1 : 1;
    }
    for (int d = 0; d < 3; ++d) {
        const int32_t x = (a[d] >> 3) & 15, y = (b[d] >> 3) & 15;
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

void hnso_sort_leaves_nanovdb(int32_t* leaf_origins, int64_t num_leaves) {
    qsort(leaf_origins, (size_t)num_leaves, sizeof(int32_t) * 3, cmp_leaf);
}

/* ---- kernels in float and in double ---------------------------------------------------- */
#define R float
#define S _f32
#define FMA fmaf
#define SQRT sqrtf
#define INV6 0.166666667f
#define OMEGA_OF_DX(dx) (2.0f / (1.0f + sinf(3.14159f * (dx))))
#include "hns_oracle_impl.h"
#undef R
#undef S
#undef FMA
#undef SQRT
#undef INV6
#undef OMEGA_OF_DX

#define R double
#define S _f64
#define FMA fma
#define SQRT sqrt
#define INV6 (1.0 / 6.0)
#define OMEGA_OF_DX(dx) (2.0 / (1.0 + sin(3.14159 * (dx))))
#include "hns_oracle_impl.h"
#undef R
#undef S
#undef FMA
#undef SQRT
#undef INV6

/* ---- HNS_Advance ------------------------------------------------------------------------
 * The reference's step is the force model's zero value (hns_oracle_impl.h,
 * hnso_hns_advance_model). */
void hnso_hns_advance_f32(const hnso_topo* t, const hnso_advance_fields* F, float dx, int iteration, float dt,
                          const hnso_combustion_params* P) {
    hnso_hns_advance_model_f32(t, F, dx, iteration, dt, P, NULL);
}
