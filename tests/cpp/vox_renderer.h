// vox_renderer.h - a header-only stand-in of the reference viewer's plugin
// interface, with the virtual signatures of vox::Renderer
// (VoxViz/VoxVizCore/Renderer.h:64-79) and the vox::Camera accessors the
// GigaVoxels renderer reads (VoxViz/VoxVizCore/Camera.h:82-109), so that the
// adapter a maintainer would add to the reference compiles and runs here.
#pragma once

#include <cstddef>
#include <string>

namespace vox {

struct Vec3 {
    float v[3];
    float x() const { return v[0]; }
    float y() const { return v[1]; }
    float z() const { return v[2]; }
};

class Camera {
public:
    Vec3 position{}, look{}, up{};
    float fov = 45.0f, near_dist = 0.1f;
    int width = 0, height = 0;
    size_t frame = 0;
    virtual ~Camera() = default;
    virtual Vec3 getPosition() const { return position; }
    const Vec3& getLook() const { return look; }
    const Vec3& getUp() const { return up; }
    float getFieldOfView() const { return fov; }
    float getNearPlaneDist() const { return near_dist; }
    void getViewportWidthHeight(int& w, int& h) const {
        w = width;
        h = height;
    }
    size_t getFrameCount() const { return frame; }
};

class SceneObject {
public:
    std::string file;  // the dataset the viewer opened
    virtual ~SceneObject() = default;
};

class Renderer {
public:
    explicit Renderer(const std::string& algorithm) : algorithm_(algorithm) {}
    virtual ~Renderer() = default;
    virtual bool acceptsFileExtension(const std::string& ext) const { return false; }
    virtual void setup() {}
    virtual void init(Camera& camera, SceneObject& scene) {}
    virtual void draw(Camera& camera, SceneObject& scene) = 0;
    virtual void update(Camera& camera, SceneObject& scene) {}
    virtual void postDraw(Camera& camera, SceneObject& scene) {}
    virtual void shutdown() {}
    const std::string& algorithm() const { return algorithm_; }

private:
    std::string algorithm_;
};

}  // namespace vox
