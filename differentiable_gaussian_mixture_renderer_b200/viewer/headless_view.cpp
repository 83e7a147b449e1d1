// Headless viewer: renders a Gaussian mixture from a camera with one of the
// three renderers through the C++ viewer interface (include/dgmr_b200_sibr.hpp),
// the reference viewer plugin's role (src/dgmr/sibr_interfaces.cpp:26-44)
// without a window: the frame goes to a PPM image and/or a raw float file.
//
//   dgmr_headless_view --scene S --camera C [--renderer splat|march|raster]
//       [--frames K] [--ppm out.ppm] [--raw out.f32] [--background r,g,b]
//       [--formulation opacity|mass|density|ots|ols] [--mode full|bins|depth]
//       [--bin B] [--max-depth D]
//
// Scene file (little endian): "DGMRSCN1", int32 n, sh_stride, sh_degree,
// reserved, then float32 centroids[n,3], sh[n,sh_stride,3], weights[n],
// scales[n,3], rotations[n,4] (w,x,y,z).
// Camera file: "DGMRCAM1", int32 width, height, then float32 view[16],
// proj[16] (glm order, proj = full view-projection), campos[3], tan_fovx,
// tan_fovy.
// Raw output: float32 [3,H,W].  Prints one line with the frame count, the
// mean milliseconds per frame (CUDA events around K frames) and the pair count.
#include "dgmr_b200_sibr.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

int usage(const char* msg)
{
    if (msg)
        std::fprintf(stderr, "dgmr_headless_view: %s\n", msg);
    std::fprintf(msg ? stderr : stdout,
        "usage: dgmr_headless_view --scene S --camera C [--renderer splat|march|raster] [--frames K]\n"
        "       [--ppm out.ppm] [--raw out.f32] [--background r,g,b] [--formulation opacity|mass|density|ots|ols]\n"
        "       [--mode full|bins|depth] [--bin B] [--max-depth D]\n");
    return msg ? 2 : 0;
}

struct HostScene {
    int32_t n = 0, sh_stride = 0, sh_degree = 0;
    std::vector<float> centroids, sh, weights, scales, rotations;
};

struct HostCamera {
    int32_t width = 0, height = 0;
    float view[16], proj[16], campos[3], tan_fovx = 0, tan_fovy = 0;
};

bool read_exact(std::FILE* f, void* dst, size_t bytes) { return std::fread(dst, 1, bytes, f) == bytes; }

bool load_scene(const char* path, HostScene* s, std::string* err)
{
    std::FILE* f = std::fopen(path, "rb");
    if (!f) {
        *err = std::string("cannot open scene ") + path;
        return false;
    }
    char magic[8];
    int32_t head[4];
    bool ok = read_exact(f, magic, 8) && std::memcmp(magic, "DGMRSCN1", 8) == 0 && read_exact(f, head, sizeof(head));
    if (ok) {
        s->n = head[0];
        s->sh_stride = head[1];
        s->sh_degree = head[2];
        ok = s->n >= 0 && s->sh_stride >= 1 && s->sh_stride <= 16 && s->sh_degree >= 0 && s->sh_degree <= 3;
    }
    if (ok) {
        const size_t n = size_t(s->n);
        s->centroids.resize(n * 3);
        s->sh.resize(n * size_t(s->sh_stride) * 3);
        s->weights.resize(n);
        s->scales.resize(n * 3);
        s->rotations.resize(n * 4);
        for (std::vector<float>* v : { &s->centroids, &s->sh, &s->weights, &s->scales, &s->rotations })
            ok = ok && read_exact(f, v->data(), v->size() * sizeof(float));
    }
    std::fclose(f);
    if (!ok)
        *err = std::string("malformed scene file ") + path;
    return ok;
}

bool load_camera(const char* path, HostCamera* c, std::string* err)
{
    std::FILE* f = std::fopen(path, "rb");
    if (!f) {
        *err = std::string("cannot open camera ") + path;
        return false;
    }
    char magic[8];
    int32_t wh[2];
    bool ok = read_exact(f, magic, 8) && std::memcmp(magic, "DGMRCAM1", 8) == 0 && read_exact(f, wh, sizeof(wh)) && read_exact(f, c->view, 64)
        && read_exact(f, c->proj, 64) && read_exact(f, c->campos, 12) && read_exact(f, &c->tan_fovx, 4) && read_exact(f, &c->tan_fovy, 4);
    std::fclose(f);
    if (ok) {
        c->width = wh[0];
        c->height = wh[1];
        ok = c->width > 0 && c->height > 0 && c->width <= 16384 && c->height <= 16384;
    }
    if (!ok)
        *err = std::string("malformed camera file ") + path;
    return ok;
}

bool parse_floats(const char* text, float* out, int n)
{
    const char* p = text;
    for (int i = 0; i < n; ++i) {
        char* end = nullptr;
        out[i] = std::strtof(p, &end);
        if (end == p)
            return false;
        p = end;
        if (i + 1 < n) {
            if (*p != ',')
                return false;
            ++p;
        }
    }
    return *p == '\0';
}

bool write_ppm(const char* path, const std::vector<float>& fb, int w, int h)
{
    std::FILE* f = std::fopen(path, "wb");
    if (!f)
        return false;
    std::fprintf(f, "P6\n%d %d\n255\n", w, h);
    std::vector<unsigned char> row(size_t(w) * 3);
    const size_t plane = size_t(w) * h;
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            for (int c = 0; c < 3; ++c) {
                float v = fb[c * plane + size_t(y) * w + x];
                v = std::isnan(v) ? 0.f : (v < 0.f ? 0.f : (v > 1.f ? 1.f : v));
                row[size_t(x) * 3 + c] = static_cast<unsigned char>(std::lround(v * 255.f));
            }
        }
        std::fwrite(row.data(), 1, row.size(), f);
    }
    return std::fclose(f) == 0;
}

template <class T>
T* upload(const std::vector<T>& v)
{
    T* d = nullptr;
    dgmr_b200::detail::check_cuda(cudaMalloc(&d, v.empty() ? sizeof(T) : v.size() * sizeof(T)), "scene upload");
    if (!v.empty())
        dgmr_b200::detail::check_cuda(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "scene upload");
    return d;
}

} // namespace

int main(int argc, char** argv)
{
    const char *scene_path = nullptr, *camera_path = nullptr, *ppm = nullptr, *raw = nullptr;
    std::string renderer = "splat", mode = "full";
    int frames = 1, bin = -1;
    float background[3] = { 0.f, 0.f, 0.f }, max_depth = 20.f;
    dgmr_formulation formulation = DGMR_FORMULATION_DEFAULT;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--help" || a == "-h")
            return usage(nullptr);
        if (i + 1 >= argc)
            return usage(("missing value after " + a).c_str());
        const char* v = argv[++i];
        if (a == "--scene")
            scene_path = v;
        else if (a == "--camera")
            camera_path = v;
        else if (a == "--renderer")
            renderer = v;
        else if (a == "--frames")
            frames = std::atoi(v);
        else if (a == "--ppm")
            ppm = v;
        else if (a == "--raw")
            raw = v;
        else if (a == "--mode")
            mode = v;
        else if (a == "--bin")
            bin = std::atoi(v);
        else if (a == "--max-depth")
            max_depth = std::strtof(v, nullptr);
        else if (a == "--background") {
            if (!parse_floats(v, background, 3))
                return usage("--background takes r,g,b");
        } else if (a == "--formulation") {
            const std::string f = v;
            const char* names[] = { "opacity", "mass", "density", "ots", "ols" };
            int code = 0;
            for (int k = 0; k < 5; ++k)
                if (f == names[k])
                    code = k + 1;
            if (code == 0)
                return usage("unknown formulation");
            formulation = dgmr_formulation(code);
        } else
            return usage(("unknown option " + a).c_str());
    }
    if (!scene_path || !camera_path)
        return usage("--scene and --camera are required");
    if (renderer != "splat" && renderer != "march" && renderer != "raster")
        return usage("--renderer must be splat, march or raster");
    if (mode != "full" && mode != "bins" && mode != "depth")
        return usage("--mode must be full, bins or depth");
    if (frames < 1 || frames > 100000)
        return usage("--frames must be in 1..100000");

    HostScene hs;
    HostCamera hc;
    std::string err;
    if (!load_scene(scene_path, &hs, &err) || !load_camera(camera_path, &hc, &err)) {
        std::fprintf(stderr, "dgmr_headless_view: %s\n", err.c_str());
        return 2;
    }

    try {
        float* d_centroids = upload(hs.centroids);
        float* d_sh = upload(hs.sh);
        float* d_weights = upload(hs.weights);
        float* d_scales = upload(hs.scales);
        float* d_rotations = upload(hs.rotations);
        float* d_fb = nullptr;
        const size_t fb_floats = size_t(3) * hc.width * hc.height;
        dgmr_b200::detail::check_cuda(cudaMalloc(&d_fb, fb_floats * sizeof(float)), "framebuffer");

        auto fill = [&](dgmr_b200::MixtureAndCamera& d) {
            d.gm_centroids = d_centroids;
            d.gm_sh_params = d_sh;
            d.gm_weights = d_weights;
            d.gm_cov_scales = d_scales;
            d.gm_cov_rotations = d_rotations;
            d.n_gaussians = hs.n;
            d.sh_stride = hs.sh_stride;
            d.sh_degree = hs.sh_degree;
            std::memcpy(d.view_matrix, hc.view, sizeof(hc.view));
            std::memcpy(d.proj_matrix, hc.proj, sizeof(hc.proj));
            std::memcpy(d.cam_poition, hc.campos, sizeof(hc.campos));
            std::memcpy(d.background, background, sizeof(background));
            d.tan_fovx = hc.tan_fovx;
            d.tan_fovy = hc.tan_fovy;
            d.formulation = formulation;
        };
        const dgmr_b200::RenderMode rm = mode == "full" ? dgmr_b200::RenderMode::Full
            : mode == "bins"                            ? dgmr_b200::RenderMode::Bins
                                                        : dgmr_b200::RenderMode::Depth;
        const dgmr_b200::Framebuffer fb { d_fb, hc.height, hc.width };
        dgmr_b200::SplatForwardData sd;
        dgmr_b200::VolMarcherForwardData md;
        dgmr_b200::VolRasterForwardData rd;
        fill(sd);
        fill(md);
        fill(rd);
        sd.framebuffer = fb;
        rd.framebuffer = fb;
        md.debug_render_mode = rd.debug_render_mode = rm;
        md.debug_render_bin = rd.debug_render_bin = bin;
        md.max_depth = rd.max_depth = max_depth;

        auto frame = [&]() -> dgmr_b200::Statistics {
            if (renderer == "splat")
                return dgmr_b200::sibr_interfaces::splat(sd);
            if (renderer == "march")
                return dgmr_b200::sibr_interfaces::vol_march(fb, md);
            return dgmr_b200::sibr_interfaces::vol_raster(rd);
        };
        dgmr_b200::Statistics st = frame(); // grows the workspaces
        cudaEvent_t t0, t1;
        dgmr_b200::detail::check_cuda(cudaEventCreate(&t0), "events");
        dgmr_b200::detail::check_cuda(cudaEventCreate(&t1), "events");
        dgmr_b200::detail::check_cuda(cudaEventRecord(t0, nullptr), "events");
        for (int k = 0; k < frames; ++k)
            st = frame();
        dgmr_b200::detail::check_cuda(cudaEventRecord(t1, nullptr), "events");
        dgmr_b200::detail::check_cuda(cudaEventSynchronize(t1), "events");
        float ms = 0.f;
        dgmr_b200::detail::check_cuda(cudaEventElapsedTime(&ms, t0, t1), "events");

        std::vector<float> host(fb_floats);
        dgmr_b200::detail::check_cuda(cudaMemcpy(host.data(), d_fb, fb_floats * sizeof(float), cudaMemcpyDeviceToHost), "framebuffer read");
        std::printf("renderer=%s frames=%d ms_per_frame=%.4f n_pairs=%u flags=%u width=%d height=%d\n", renderer.c_str(), frames, ms / frames,
            st.n_pairs, st.flags, hc.width, hc.height);
        if (raw) {
            std::FILE* f = std::fopen(raw, "wb");
            if (!f || std::fwrite(host.data(), sizeof(float), host.size(), f) != host.size() || std::fclose(f) != 0) {
                std::fprintf(stderr, "dgmr_headless_view: cannot write %s\n", raw);
                return 1;
            }
        }
        if (ppm && !write_ppm(ppm, host, hc.width, hc.height)) {
            std::fprintf(stderr, "dgmr_headless_view: cannot write %s\n", ppm);
            return 1;
        }
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        for (void* p : { (void*)d_centroids, (void*)d_sh, (void*)d_weights, (void*)d_scales, (void*)d_rotations, (void*)d_fb })
            cudaFree(p);
    } catch (const dgmr_b200::Error& e) {
        std::fprintf(stderr, "dgmr_headless_view: %s\n", e.what());
        return 1;
    }
    return 0;
}
