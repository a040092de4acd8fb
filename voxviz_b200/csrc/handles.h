// handles.h - the structs behind the opaque C handles vv_octree and
// vv_renderer, shared by the C ABI and the paged scene.
#pragma once

#include <memory>

#include "ctx.h"
#include "octree.h"
#include "renderer.h"

struct vv_octree {
    std::shared_ptr<const vv::TerrainVolume> volume;  // terrain trees only
    std::unique_ptr<vv::GigaVoxelsOctTree> tree;
};

struct vv_renderer {
    std::unique_ptr<vv::GigaVoxelsRenderer> impl;
    vv_ctx* ctx = nullptr;
};
