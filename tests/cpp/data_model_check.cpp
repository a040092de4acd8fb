// data_model_check.cpp - drives the C++ data-model API of voxviz_b200.hpp
// and the vox::Renderer adapter; prints one JSON object per check.
//
//   layout  <depth> <collapse>          OctTreeNodePool rebuilt from a terrain
//                                       octree lays out the same node words
//   paging  <depth> <cams> <bricks>     host data model (OctTreeNodePool +
//                                       BrickPool::processNodeUsageList/update)
//                                       against the library's renderer, frame
//                                       by frame (needs a GPU)
//   adapter <depth> <cams>              the vox::Renderer plugin against the
//                                       library's renderer (needs a GPU)
// <cams>: a file of vv_camera records.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "gigavoxels_b200_adapter.h"

static vv_terrain_desc terrain(int depth, int collapse) {
    return vv_terrain_desc{3u, depth, 4, 2.0f, 0.5f, 4, collapse, 0};
}

static std::vector<vv_camera> read_cams(const char* path) {
    std::vector<vv_camera> cams;
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error("cannot open the camera file");
    vv_camera c;
    while (std::fread(&c, sizeof(c), 1, f) == 1) cams.push_back(c);
    std::fclose(f);
    return cams;
}

static int layout(int depth, int collapse) {
    vv::GigaVoxelsOctTree t = vv::GigaVoxelsOctTree::build(terrain(depth, collapse));
    vv::OctTreeNodePool pool = vv::OctTreeNodePool::fromOctree(t);
    const std::vector<uint32_t> w = pool.create3DTexture();
    size_t dx, dy, dz;
    pool.get3DTextureDimensions(dx, dy, dz);
    const std::vector<uint32_t> ref = t.nodeWords();
    const bool dims = (int)dx == t.info().pool_dim[0] && (int)dy == t.info().pool_dim[1] &&
                      (int)dz == t.info().pool_dim[2];
    std::printf("{\"check\": \"layout\", \"depth\": %d, \"collapse\": %d, \"nodes\": %zu, \"dims_equal\": %s, "
                "\"words_equal\": %s, \"levels\": %d}\n",
                depth, collapse, pool.getNodeCount(), dims ? "true" : "false",
                (dims && w == ref) ? "true" : "false", t.getDepth());
    return 0;
}

static void download(vv_ctx* c, std::vector<uint32_t>& w, size_t n) {
    w.assign(n, 0u);
    vv::check(vv_nodepool_download(c, 0, w.data()), "download", c);
}

static int paging(int depth, const char* cam_path, int bricks) {
    const std::vector<vv_camera> cams = read_cams(cam_path);
    vv::GigaVoxelsOctTree t = vv::GigaVoxelsOctTree::build(terrain(depth, 1));
    // the library's renderer: device LRU, device brick production
    vv_params p{};
    vv_ctx* cb = nullptr;
    vv::check(vv_ctx_create(&p, &cb), "ctx");
    vv_renderer_desc d{};
    d.fmt = VV_FMT_RGBA8;
    d.pool_bytes = (int64_t)bricks * 4000;
    d.lod_scalar = 1.0f;
    d.alpha_stop = 0.99f;
    d.jitter_seed = 7;
    d.device_paging = 1;
    vv_renderer* rb = nullptr;
    vv::check(vv_renderer_create(cb, t.handle(), &d, &rb), "renderer", cb);
    // the host data model on its own context
    vv_ctx* ca = nullptr;
    vv::check(vv_ctx_create(&p, &ca), "ctx");
    vv::OctTreeNodePool pool = vv::OctTreeNodePool::fromOctree(t);
    pool.create3DTexture(ca, 0);
    vv::BrickPool& bp = vv::BrickPool::instance();
    bp.init(ca, 8, 8, 8, (size_t)bricks);
    std::vector<uint8_t> jit(32 * 32);
    vv::check(vv_make_jitter(7, 32, jit.data()), "jitter");
    vv::check(vv_set_jitter(ca, jit.data(), 32), "jitter", ca);
    // the root brick (initBricks of the reference): as the renderer's init
    if (!pool.getChild(0)->isConstant()) {
        bp.getUploadRequestList().push_back(0);
        bp.update(t, pool);
        pool.update();
    }
    size_t dx, dy, dz;
    pool.get3DTextureDimensions(dx, dy, dz);
    const size_t words = dx * dy * dz * 2;
    int32_t slots[3], fmt;
    vv::check(vv_brickpool_info(ca, slots, &fmt), "pool info", ca);
    int equal_frames = 0, evictions = 0;
    size_t requests_total = 0;
    for (const vv_camera& cam : cams) {
        // B: draw, postDraw and update through the renderer's frame protocol
        vv::check(vv_renderer_draw_passes(rb, &cam, VV_PASS_RAYCAST), "draw", cb);
        vv::check(vv_renderer_post_draw(rb), "postDraw", cb);
        vv::check(vv_renderer_update(rb), "update", cb);
        // A: the ray cast and the three passes, then the host data model
        vv_uniforms u;
        vv::check(vv_compute_uniforms(&t.info(), &cam, slots[0], slots[1], slots[2], 1.0f, 0.99f, &u), "uniforms");
        const size_t np = (size_t)cam.width * cam.height;
        uint32_t *req = nullptr, *cnt = nullptr;
        if (cudaMalloc((void**)&req, np * 16) != cudaSuccess || cudaMalloc((void**)&cnt, 4) != cudaSuccess)
            throw std::runtime_error("cudaMalloc");
        vv_frame_out o{};
        o.requests = req;
        o.request_count = cnt;
        o.request_cap = (int32_t)np;
        o.compress_max_push = 4 * (cam.frame % 3 + 1);
        o.passes = VV_PASS_ALL;
        vv::check(vv_render(ca, 0, &u, &o), "render", ca);
        uint32_t n = 0;
        cudaMemcpy(&n, cnt, 4, cudaMemcpyDeviceToHost);
        n = std::min<uint32_t>(n, (uint32_t)np);
        std::vector<uint32_t> h((size_t)n * 4);
        if (n) cudaMemcpy(h.data(), req, (size_t)n * 16, cudaMemcpyDeviceToHost);
        cudaFree(req);
        cudaFree(cnt);
        requests_total += n;
        bp.processNodeUsageList(h.data(), n, pool);
        bp.update(t, pool);
        pool.update();
        // compare: requests, residency, LRU order, node words
        int32_t nb = 0;
        vv::check(vv_renderer_last_requests(rb, nullptr, 0, &nb), "requests", cb);
        std::vector<uint32_t> hb((size_t)nb * 4);
        vv::check(vv_renderer_last_requests(rb, hb.data(), nb, &nb), "requests", cb);
        int64_t nr = 0;
        vv::check(vv_renderer_residency(rb, nullptr, nullptr, 0, &nr), "residency", cb);
        std::vector<uint32_t> rxyz((size_t)nr * 3), rslot((size_t)nr);
        vv::check(vv_renderer_residency(rb, rxyz.data(), rslot.data(), nr, &nr), "residency", cb);
        std::map<size_t, size_t> ra, rbm;
        for (const auto& e : bp.residency()) ra[e.second] = e.first;
        for (int64_t k = 0; k < nr; ++k)
            rbm[rslot[(size_t)k]] = pool.nodeIndexAt(rxyz[3 * k], rxyz[3 * k + 1], rxyz[3 * k + 2]);
        int64_t no = 0;
        vv::check(vv_renderer_lru_order(rb, nullptr, 0, &no), "lru", cb);
        std::vector<uint32_t> lb((size_t)no);
        vv::check(vv_renderer_lru_order(rb, lb.data(), no, &no), "lru", cb);
        std::vector<uint32_t> wa, wb;
        download(ca, wa, words);
        download(vv_renderer_ctx(rb), wb, words);
        vv_renderer_stats st;
        vv_renderer_get_stats(rb, &st);
        evictions = (int)st.evictions_total;
        const bool same = h == hb && ra == rbm && bp.lruOrder() == lb && wa == wb;
        std::printf("{\"check\": \"paging\", \"frame\": %d, \"requests\": %u, \"resident\": %zu, "
                    "\"requests_equal\": %s, \"residency_equal\": %s, \"lru_equal\": %s, \"words_equal\": %s}\n",
                    cam.frame, n, ra.size(), h == hb ? "true" : "false", ra == rbm ? "true" : "false",
                    bp.lruOrder() == lb ? "true" : "false", wa == wb ? "true" : "false");
        if (!same) break;
        ++equal_frames;
    }
    std::printf("{\"check\": \"paging_summary\", \"frames\": %zu, \"equal_frames\": %d, \"evictions\": %d, "
                "\"requests\": %zu, \"uploaded\": %zu}\n",
                cams.size(), equal_frames, evictions, requests_total, bp.getNumBricksUploaded());
    bp.reset();
    vv_renderer_destroy(rb);
    vv_ctx_destroy(cb);
    vv_ctx_destroy(ca);
    return 0;
}

static int adapter(int depth, const char* cam_path) {
    const std::vector<vv_camera> cams = read_cams(cam_path);
    vv_renderer_desc d{};
    d.fmt = VV_FMT_RGBA8;
    d.pool_bytes = 400ll * 4000;
    d.lod_scalar = 1.0f;
    d.alpha_stop = 0.99f;
    d.jitter_seed = 7;
    d.device_paging = 1;
    // the plugin, driven as the viewer drives it (GLWidget: draw, postDraw, update)
    GigaVoxelsB200Renderer plugin;
    plugin.terrain = terrain(depth, 1);
    plugin.desc = d;
    vox::Renderer* r = &plugin;
    vox::SceneObject scene;
    vox::Camera vc;
    r->init(vc, scene);
    // the library's renderer directly
    vv::GigaVoxelsOctTree t = vv::GigaVoxelsOctTree::build(terrain(depth, 1));
    vv_params p{};
    vv_ctx* c = nullptr;
    vv::check(vv_ctx_create(&p, &c), "ctx");
    vv_renderer* rr = nullptr;
    vv::check(vv_renderer_create(c, t.handle(), &d, &rr), "renderer", c);
    int equal = 0;
    for (const vv_camera& cam : cams) {
        for (int a = 0; a < 3; ++a) {
            vc.position.v[a] = cam.position[a];
            vc.look.v[a] = cam.look[a];
            vc.up.v[a] = cam.up[a];
        }
        vc.fov = cam.fov_y_deg;
        vc.near_dist = cam.near_dist;
        vc.width = cam.width;
        vc.height = cam.height;
        vc.frame = (size_t)cam.frame;
        r->draw(vc, scene);
        std::vector<float> ca((size_t)cam.width * cam.height * 4), cb(ca.size());
        vv::check(vv_renderer_read_color(plugin.renderer().handle(), ca.data()), "read", nullptr);
        r->postDraw(vc, scene);
        r->update(vc, scene);
        vv::check(vv_renderer_draw(rr, &cam), "draw", c);
        vv::check(vv_renderer_read_color(rr, cb.data()), "read", c);
        vv::check(vv_renderer_update(rr), "update", c);
        vv_renderer_stats sa, sb;
        vv_renderer_get_stats(plugin.renderer().handle(), &sa);
        vv_renderer_get_stats(rr, &sb);
        const bool same = ca == cb && sa.requests == sb.requests && sa.bricks_uploaded == sb.bricks_uploaded &&
                          sa.resident_bricks == sb.resident_bricks;
        if (!same) break;
        ++equal;
    }
    std::printf("{\"check\": \"adapter\", \"frames\": %zu, \"equal_frames\": %d, \"algorithm\": \"%s\"}\n",
                cams.size(), equal, r->algorithm().c_str());
    r->shutdown();
    vv_renderer_destroy(rr);
    vv_ctx_destroy(c);
    return 0;
}

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "layout" && argc == 4) return layout(std::atoi(argv[2]), std::atoi(argv[3]));
        if (mode == "paging" && argc == 5) return paging(std::atoi(argv[2]), argv[3], std::atoi(argv[4]));
        if (mode == "adapter" && argc == 4) return adapter(std::atoi(argv[2]), argv[3]);
        std::fprintf(stderr, "usage: layout <depth> <collapse> | paging <depth> <cams> <bricks> | adapter <depth> <cams>\n");
        return 2;
    } catch (const vv::Error& e) {
        std::fprintf(stderr, "vv::Error %d: %s\n", e.code(), e.what());
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
