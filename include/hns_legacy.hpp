// hns_legacy.hpp -- the reference's own C++ entry points for the solver path, re-implemented
// over the C ABI of hns.h (libhns.so exports both).
//
// A SOP written against the reference binds these names and signatures:
//   src/Cuda/HNanoSolver.cu:51-515   HNS_EnsureContext, HNS_UploadSources, HNS_Advance,
//                                    HNS_DownloadForOutput, HNS_GetActiveMask,
//                                    HNS_DestroyContext, CreateIndexGrid, Compute_Sim
//   src/SOP/Advection/SOP_VDBAdvect.hpp:66                     AdvectIndexGrid
//   src/SOP/VelocityAdvection/SOP_VDBAdvectVelocity.hpp:60     AdvectIndexGridVelocity
//   src/SOP/ProjectNonDivergent/SOP_VDBProjectNonDivergent.hpp:69-70
//                                                    ProjectNonDivergent, Divergence
// Differences a caller sees: HNS::GridIndexedData here stores its own POD Coord/Vec3f
// (layout-identical to openvdb::Coord / openvdb::Vec3f, so a SOP can reinterpret_cast its
// OpenVDB buffers), and CreateIndexGrid fills an HNS::IndexGridHandle (the leaf table)
// instead of a nanovdb::GridHandle<nanovdb::cuda::DeviceBuffer>. As in the reference,
// failures throw std::runtime_error.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <typeindex>
#include <unordered_map>
#include <vector>

#include "hns.h"

// Same layout as the reference's CombustionParams (src/Cuda/Kernels.cuh:5-24).
typedef hns_combustion_params CombustionParams;

enum class AllocationType { Standard, Aligned, CudaPinned };

namespace HNS {

struct Coord {
    int32_t x, y, z;
    int32_t operator[](int i) const { return (&x)[i]; }
};

struct Vec3f {
    float x, y, z;
    float operator[](int i) const { return (&x)[i]; }
};

static_assert(sizeof(Coord) == 12 && sizeof(Vec3f) == 12, "POD layout of openvdb::Coord / Vec3f");

// Host SoA container of the indexed layout (src/Utils/GridData.hpp:16-166): one coordinate
// block plus named typed value blocks, all of size() elements, in slot order.
class GridIndexedData {
   public:
    GridIndexedData() = default;
    GridIndexedData(const GridIndexedData&) = delete;
    GridIndexedData& operator=(const GridIndexedData&) = delete;
    GridIndexedData(GridIndexedData&&) = default;
    GridIndexedData& operator=(GridIndexedData&&) = default;
    ~GridIndexedData() { clear(); }

    bool allocateCoords(size_t numElements) {
        m_coords = Block(numElements * sizeof(Coord), m_allocType);
        if (numElements && !m_coords.ptr) return false;
        m_size = numElements;
        return true;
    }

    template <typename T>
    bool addValueBlock(const std::string& name, size_t numElements) {
        if (m_index.count(name)) return false;
        Entry e{name, std::type_index(typeid(T)), Block(numElements * sizeof(T), m_allocType)};
        if (numElements && !e.block.ptr) return false;
        m_blocks.push_back(std::move(e));
        m_index[name] = m_blocks.size() - 1;
        return true;
    }

    template <typename T>
    T* pValues(const std::string& name) {
        auto it = m_index.find(name);
        if (it == m_index.end() || m_blocks[it->second].type != std::type_index(typeid(T))) return nullptr;
        return static_cast<T*>(m_blocks[it->second].block.ptr);
    }

    template <typename T>
    const T* pValues(const std::string& name) const {
        return const_cast<GridIndexedData*>(this)->pValues<T>(name);
    }

    Coord* pCoords() { return static_cast<Coord*>(m_coords.ptr); }
    const Coord* pCoords() const { return static_cast<const Coord*>(m_coords.ptr); }
    size_t size() const { return m_size; }
    size_t numValueBlocks() const { return m_blocks.size(); }

    template <typename T>
    std::vector<std::string> getBlocksOfType() const {
        std::vector<std::string> names;
        for (const auto& e : m_blocks)
            if (e.type == std::type_index(typeid(T))) names.push_back(e.name);
        return names;
    }

    void clearValues() {
        m_blocks.clear();
        m_index.clear();
    }
    void clear() {
        clearValues();
        m_coords = Block();
        m_size = 0;
    }
    void setAllocationType(AllocationType t) { m_allocType = t; }

   private:
    // Standard (new[]), 64-byte aligned, or CUDA pinned host memory
    // (src/Utils/Memory.hpp:37-111).
    struct Block {
        void* ptr = nullptr;
        AllocationType type = AllocationType::Standard;
        Block() = default;
        Block(size_t bytes, AllocationType t) : type(t) {
            if (!bytes) return;
            if (t == AllocationType::CudaPinned) {
                if (cudaMallocHost(&ptr, bytes) != cudaSuccess) ptr = nullptr;
            } else if (t == AllocationType::Aligned) {
                ptr = ::operator new(bytes, std::align_val_t(64), std::nothrow);
            } else {
                ptr = ::operator new(bytes, std::nothrow);
            }
            if (ptr) std::memset(ptr, 0, bytes);
        }
        Block(const Block&) = delete;
        Block& operator=(const Block&) = delete;
        Block(Block&& o) noexcept : ptr(o.ptr), type(o.type) { o.ptr = nullptr; }
        Block& operator=(Block&& o) noexcept {
            if (this != &o) {
                release();
                ptr = o.ptr, type = o.type;
                o.ptr = nullptr;
            }
            return *this;
        }
        ~Block() { release(); }
        void release() {
            if (!ptr) return;
            if (type == AllocationType::CudaPinned)
                (void)cudaFreeHost(ptr);
            else if (type == AllocationType::Aligned)
                ::operator delete(ptr, std::align_val_t(64));
            else
                ::operator delete(ptr);
            ptr = nullptr;
        }
    };
    struct Entry {
        std::string name;
        std::type_index type;
        Block block;
    };
    Block m_coords;
    std::vector<Entry> m_blocks;
    std::unordered_map<std::string, size_t> m_index;
    size_t m_size = 0;
    AllocationType m_allocType = AllocationType::Standard;
};

// What CreateIndexGrid produces: the domain's leaves in slot order and the voxel size (the
// reference's handle owns a device NanoVDB ValueOnIndex grid; libhns builds its leaf
// tables from this inside the context).
struct IndexGridHandle {
    std::vector<int32_t> leafOrigins;  // 3 per leaf
    float voxelSize = 0.f;
    size_t numVoxels() const { return leafOrigins.size() / 3 * 512; }
    bool empty() const { return leafOrigins.empty(); }
};

}  // namespace HNS

extern "C" {
// Builds the index grid of data's leaf-dense coordinates (src/Cuda/HNanoSolver.cu:507-510).
HNS_API void CreateIndexGrid(HNS::GridIndexedData& data, HNS::IndexGridHandle& handle, float voxelSize);
// (src/Cuda/HNanoSolver.cu:58-156) Creates the context when *ctx is null or N / voxelSize
// changed, uploading the velocity ("velocity" or the first Vec3f block) and every float
// block except src_* and collision_sdf; otherwise keeps the device state and only refreshes
// the grid. hasCollision uploads "collision_sdf" when present (stored, not used: the
// collision branches are outside this solver's scope).
HNS_API void HNS_EnsureContext(void** ctx, HNS::GridIndexedData& data, const HNS::IndexGridHandle& handle,
                               float voxelSize, bool hasCollision);
// (src/Cuda/HNanoSolver.cu:158-221) Replaces the sources with data's src_vel (Vec3f) or
// src_vel_x/y/z and every src_* float block.
HNS_API void HNS_UploadSources(void* ctx, HNS::GridIndexedData& data);
// (src/Cuda/HNanoSolver.cu:223-456) One frame; a null context is a no-op.
HNS_API void HNS_Advance(void* ctx, int iteration, float dt, const CombustionParams& params);
// (src/Cuda/HNanoSolver.cu:471-495) Velocity into data's velocity block, every state scalar
// into the float block of the same name when data has one.
HNS_API void HNS_DownloadForOutput(void* ctx, HNS::GridIndexedData& data);
// (src/Cuda/HNanoSolver.cu:459-468)
HNS_API void HNS_GetActiveMask(void* ctx, std::vector<unsigned char>& hostMask);
// (src/Cuda/HNanoSolver.cu:51-56)
HNS_API void HNS_DestroyContext(void** ctx);
// (src/Cuda/HNanoSolver.cu:512-515) An empty stub in the reference; kept for link parity.
HNS_API void Compute_Sim(HNS::GridIndexedData& data, const HNS::IndexGridHandle& handle, int iteration, float dt,
                         float voxelSize, const CombustionParams& params, bool hasCollision, const cudaStream_t& stream);

// HNanoAdvect: every float block advected, in place, by the single Vec3f block
// (advect_scalar semantics; src/Cuda/Advection.cu:13-112, commented out in the reference).
HNS_API void AdvectIndexGrid(HNS::GridIndexedData& data, float dt, float voxelSize, const cudaStream_t& stream);
// HNanoAdvectVelocity: the single Vec3f block advected by itself, in place
// (src/Cuda/Advection.cu:114-166).
HNS_API void AdvectIndexGridVelocity(HNS::GridIndexedData& data, float dt, float voxelSize, const cudaStream_t& stream);
// HNanoProjectNonDivergent: the single Vec3f block made divergence-free in place with
// `iteration` red-black iterations (src/Cuda/PressureProjection.cu:9-78).
HNS_API void ProjectNonDivergent(HNS::GridIndexedData& data, size_t iteration, float voxelSize, const cudaStream_t& stream);
// Divergence of the single Vec3f block into the float block "divergence"
// (src/Cuda/PressureProjection.cu:81-125).
HNS_API void Divergence(HNS::GridIndexedData& data, float voxelSize, const cudaStream_t& stream);
}
