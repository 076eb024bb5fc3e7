// Metal/Metal.hpp -- inert host stand-in for the handful of metal-cpp
// declarations that the reference's ANEOS.cpp and Buffers.hpp mention, so that
// ANEOS.cpp compiles unchanged into oracle/_ref.  Only the table loader
// (loadANEOSDataFromFile) is called; the texture objects below do nothing.
// TEST INFRASTRUCTURE ONLY.
#ifndef REF_SHIM_METAL_HPP
#define REF_SHIM_METAL_HPP
#include <cstddef>
namespace MTL {
enum PixelFormat { PixelFormatRG32Float };
enum TextureUsage { TextureUsageShaderRead };
enum StorageMode { StorageModePrivate, StorageModeShared };
enum ResourceOptions { ResourceStorageModeShared, ResourceStorageModePrivate };
struct Region {
    static Region Make2D(size_t, size_t, size_t, size_t) { return Region(); }
};
struct TextureDescriptor {
    static TextureDescriptor *texture2DDescriptor(PixelFormat, size_t, size_t, bool) { return nullptr; }
    void setUsage(TextureUsage) {}
    void setStorageMode(StorageMode) {}
};
struct Texture {
    void replaceRegion(Region, size_t, const void *, size_t) {}
    void release() {}
};
struct Buffer {
    void *contents() { return nullptr; }
    void release() {}
};
struct CommandQueue {};
struct Device {
    Texture *newTexture(TextureDescriptor *) { return nullptr; }
    Buffer *newBuffer(unsigned long, ResourceOptions) { return nullptr; }
};
}  // namespace MTL
#endif
