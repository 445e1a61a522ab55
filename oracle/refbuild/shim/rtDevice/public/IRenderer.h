/* oracle/refbuild/shim/rtDevice/public/IRenderer.h -- TEST INFRASTRUCTURE ONLY.
 * Stand-in for src/rtDevice/public/IRenderer.h, whose real version includes
 * <vulkan/vulkan.h>. Declares only the three buffer calls BVHGeometry uses
 * (src/Renderer/BVHGeometry.cpp:7-17,69-78); the oracle's renderer implements
 * them as host no-ops because the builder's output is read back on the CPU. */
#pragma once
#include "timCore/type.h"
#include "rtDevice/public/Resource.h"
#include "rtDevice/public/IRenderContext.h"

namespace tim
{
    class IRenderer
    {
    public:
        virtual ~IRenderer() {}
        virtual BufferHandle CreateBuffer(u32 _size, MemoryType _memType, BufferUsage _usage) = 0;
        virtual void DestroyBuffer(BufferHandle& _buffer) = 0;
        virtual void UploadBuffer(BufferHandle _handle, void* _data, u32 _dataSize) = 0;
        virtual void UploadBuffer(BufferHandle _handle, u32 _destOffset, void* _data, u32 _dataSize) = 0;
    };
}
