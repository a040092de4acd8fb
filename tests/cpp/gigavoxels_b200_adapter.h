// gigavoxels_b200_adapter.h - the "gv" vox::Renderer plugin a maintainer
// would add to the reference (GigaVoxels/GigaVoxelsB200.h), calling this
// library instead of the GLSL passes: the same frame protocol as
// GigaVoxelsRenderer (GigaVoxelsRenderer.cpp: init :341-607, draw :905-1148,
// postDraw :1150-1186, update :1520-1582), with postDraw kept apart.
#pragma once

#include <string>

#include "voxviz_b200.hpp"
#include "vox_renderer.h"

class GigaVoxelsB200Renderer : public vox::Renderer {
public:
    GigaVoxelsB200Renderer() : vox::Renderer("gv") {}
    // the dataset when the scene names none: the seeded terrain
    vv_terrain_desc terrain{1u, 5, 4, 2.0f, 0.5f, 4, 1, 0};
    vv_renderer_desc desc{};

    bool acceptsFileExtension(const std::string& ext) const override { return ext == "gvx"; }

    void init(vox::Camera&, vox::SceneObject& scene) override {
        vv::GigaVoxelsOctTree tree = scene.file.empty() ? vv::GigaVoxelsOctTree::build(terrain)
                                                        : vv::GigaVoxelsOctTree::LoadOctTreeFile(scene.file);
        r_.init(0, std::move(tree), desc);
    }
    void draw(vox::Camera& cam, vox::SceneObject&) override {
        vv_camera c{};
        const vox::Vec3 p = cam.getPosition();  // the volume box is the unit cube
        for (int a = 0; a < 3; ++a) {
            c.position[a] = p.v[a];
            c.look[a] = cam.getLook().v[a];
            c.up[a] = cam.getUp().v[a];
        }
        c.fov_y_deg = cam.getFieldOfView();
        c.near_dist = cam.getNearPlaneDist();
        cam.getViewportWidthHeight(c.width, c.height);
        c.frame = (int32_t)cam.getFrameCount();
        r_.draw(c);
    }
    void postDraw(vox::Camera&, vox::SceneObject&) override { r_.postDraw(); }
    void update(vox::Camera&, vox::SceneObject&) override { r_.update(); }
    void shutdown() override { r_.shutdown(); }

    vv::GigaVoxelsRenderer& renderer() { return r_; }

private:
    vv::GigaVoxelsRenderer r_;
};
