// es_proposal_net: the tile-proposal network on the device (no counterpart in the reference): FP32 master weights,
// their bfloat16-rounded copy used by every forward pass, Adam's moments, and the tensor-core fragments of the fused
// inference kernel. Training runs the project's own forward, backward and Adam kernels on crops of features.
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "es_internal.h"

using namespace es;

struct es_proposal_net {
    DeviceBuffer<float> params, rounded, grads, m, v;
    DeviceBuffer<uint32_t> frags;
    bool frags_current = false;
    int t = 0;
    // training scratch, sized for the largest batch seen
    int cap_n = 0, cap_h = 0, cap_w = 0;
    DeviceBuffer<float> a1, a2, a3, z, g3, g2, g1, gz, loss_parts;
    PinnedBuffer<float> h_loss;
    // es_proposal_predict's feature map and need flags, sized for the largest picture seen
    DeviceBuffer<float2> feat;
    DeviceBuffer<unsigned> need;
};

namespace {

void init_net(es_proposal_net &net, const float *host, uint64_t seed)
{
    std::vector<float> p(kNetParams, 0.0f);
    if (host) {
        std::memcpy(p.data(), host, sizeof(float) * kNetParams);
    } else {
        // He initialisation, zero biases
        std::mt19937_64 rng(seed);
        const int ci[4] = {2, 16, 16, 16}, co[4] = {16, 16, 16, 1};
        for (int l = 0; l < 4; l++) {
            std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * ci[l])));
            for (int i = 0; i < co[l] * ci[l] * 9; i++) p[net_w(l) + i] = nd(rng);
        }
    }
    std::vector<float> r(kNetParams);
    for (int i = 0; i < kNetParams; i++) {
        // round to nearest bfloat16, ties to even (finite inputs)
        uint32_t u;
        std::memcpy(&u, &p[i], 4);
        u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
        std::memcpy(&r[i], &u, 4);
    }
    net.params.reset(kNetParams);
    net.rounded.reset(kNetParams);
    net.grads.reset(kNetParams);
    net.m.reset(kNetParams);
    net.v.reset(kNetParams);
    net.frags.reset(kNetFrags);
    cuda_check(cudaMemcpy(net.params.ptr, p.data(), sizeof(float) * kNetParams, cudaMemcpyHostToDevice), "network set-up");
    cuda_check(cudaMemcpy(net.rounded.ptr, r.data(), sizeof(float) * kNetParams, cudaMemcpyHostToDevice), "network set-up");
    cuda_check(cudaMemset(net.grads.ptr, 0, sizeof(float) * kNetParams), "network set-up");
    cuda_check(cudaMemset(net.m.ptr, 0, sizeof(float) * kNetParams), "network set-up");
    cuda_check(cudaMemset(net.v.ptr, 0, sizeof(float) * kNetParams), "network set-up");
    net.t = 0;
    net.frags_current = false;
}

void ensure_scratch(es_proposal_net &net, int n, int h, int w)
{
    if (n <= net.cap_n && h == net.cap_h && w == net.cap_w) return;
    net.cap_n = n;
    net.cap_h = h;
    net.cap_w = w;
    auto plane = [&](int shrink, int ch) { return (size_t)n * ch * (h - shrink) * (w - shrink); };
    net.a1.reset(plane(2, 16));
    net.a2.reset(plane(4, 16));
    net.a3.reset(plane(6, 16));
    net.z.reset(plane(8, 1));
    net.gz.reset(plane(8, 1));
    net.g3.reset(plane(6, 16));
    net.g2.reset(plane(4, 16));
    net.g1.reset(plane(2, 16));
    const size_t tiles = (size_t)n * ((h - 8) / 16) * ((w - 8) / 16);
    net.loss_parts.reset(tiles);
    net.h_loss.reset(tiles);
}

}  // namespace

// Used by es_batch: the parameters and fragments of the inference kernel (fragments packed on first use).
const float *proposal_net_rounded(es_proposal_net *net, cudaStream_t s)
{
    if (!net->frags_current) {
        cuda_check(launch_net_pack(net->rounded.ptr, net->frags.ptr, s), "packing the network");
        net->frags_current = true;
    }
    return net->rounded.ptr;
}
const uint32_t *proposal_net_frags(const es_proposal_net *net) { return net->frags.ptr; }

extern "C" {

int es_proposal_net_create(const float *params, uint64_t seed, es_proposal_net **out)
{
    return guarded([&] {
        require(out != nullptr, "es_proposal_net_create: NULL argument");
        check_device();
        auto net = std::make_unique<es_proposal_net>();
        init_net(*net, params, seed);
        *out = net.release();
    });
}

int es_proposal_net_get(const es_proposal_net *net, float *params)
{
    return guarded([&] {
        require(net != nullptr && params != nullptr, "es_proposal_net_get: NULL argument");
        cuda_check(cudaMemcpy(params, net->params.ptr, sizeof(float) * kNetParams, cudaMemcpyDeviceToHost), "reading the network");
    });
}

int es_proposal_net_train_step(es_proposal_net *net, const float *x, const float *labels, int n, int h, int w, float lr,
                               double *loss, float *grads, void *stream)
{
    return guarded([&] {
        require(net != nullptr && x != nullptr && labels != nullptr, "es_proposal_net_train_step: NULL argument");
        require(n > 0 && h > 8 && w > 8 && (h - 8) % 16 == 0 && (w - 8) % 16 == 0,
                "es_proposal_net_train_step: crops must be 8 + 16 k feature pixels per side");
        cudaStream_t s = (cudaStream_t)stream;
        ensure_scratch(*net, n, h, w);
        const float *P = net->params.ptr;
        cuda_check(launch_net_forward(0, x, n, h, w, P, net->a1.ptr, s), "training forward");
        cuda_check(launch_net_forward(1, net->a1.ptr, n, h - 2, w - 2, P, net->a2.ptr, s), "training forward");
        cuda_check(launch_net_forward(2, net->a2.ptr, n, h - 4, w - 4, P, net->a3.ptr, s), "training forward");
        cuda_check(launch_net_forward(3, net->a3.ptr, n, h - 6, w - 6, P, net->z.ptr, s), "training forward");
        const int ta = (h - 8) / 16, tb = (w - 8) / 16;
        cuda_check(launch_net_loss(net->z.ptr, labels, n, ta, tb, net->gz.ptr, net->loss_parts.ptr, s), "training loss");
        cuda_check(launch_net_backward(3, net->gz.ptr, net->a3.ptr, n, h - 6, w - 6, P, net->g3.ptr, net->grads.ptr, s), "training backward");
        cuda_check(launch_net_backward(2, net->g3.ptr, net->a2.ptr, n, h - 4, w - 4, P, net->g2.ptr, net->grads.ptr, s), "training backward");
        cuda_check(launch_net_backward(1, net->g2.ptr, net->a1.ptr, n, h - 2, w - 2, P, net->g1.ptr, net->grads.ptr, s), "training backward");
        cuda_check(launch_net_backward(0, net->g1.ptr, x, n, h, w, P, nullptr, net->grads.ptr, s), "training backward");
        if (grads)
            cuda_check(cudaMemcpyAsync(grads, net->grads.ptr, sizeof(float) * kNetParams, cudaMemcpyDeviceToHost, s), "reading gradients");
        if (lr > 0.0f) {
            net->t++;
            cuda_check(launch_net_adam(net->params.ptr, net->rounded.ptr, net->grads.ptr, net->m.ptr, net->v.ptr, kNetParams, lr, 0.9f,
                                       0.999f, 1e-8f, net->t, s),
                       "training step");
            net->frags_current = false;
        }
        if (loss) {
            const size_t tiles = (size_t)n * ta * tb;
            cuda_check(cudaMemcpyAsync(net->h_loss.ptr, net->loss_parts.ptr, sizeof(float) * tiles, cudaMemcpyDeviceToHost, s), "reading the loss");
            cuda_check(cudaStreamSynchronize(s), "training step");
            double sum = 0.0;
            for (size_t i = 0; i < tiles; i++) sum += net->h_loss.ptr[i];
            *loss = sum / (double)tiles;
        } else if (grads) {
            cuda_check(cudaStreamSynchronize(s), "training step");
        }
    });
}

int es_proposal_features(uint64_t words, int w, int h, const int *xy, int n, int fw, int fh, float *out, void *stream)
{
    return guarded([&] {
        require(words != 0 && xy != nullptr && out != nullptr, "es_proposal_features: NULL argument");
        require(w > 0 && h > 0 && n > 0 && fw > 0 && fh > 0, "es_proposal_features: sizes must be positive");
        cuda_check(launch_net_features((const uint16_t *)words, w, h, xy, n, fw, fh, out, (cudaStream_t)stream), "features");
    });
}

int es_proposal_predict(es_proposal_net *net, uint64_t words, int w, int h, float *pred, void *stream)
{
    return guarded([&] {
        require(net != nullptr && words != 0 && pred != nullptr, "es_proposal_predict: NULL argument");
        require(w >= 2 && h >= 2, "es_proposal_predict: picture too small");
        cudaStream_t s = (cudaStream_t)stream;
        const es_cambi_params p = derive_params(w, h);
        PredBatch pb{};
        pb.njobs = 1;
        PredJob &j = pb.job[0];
        j.word = (const uint16_t *)words;
        j.w = w;
        j.h = h;
        j.tiles_x = (w + 63) / 64;
        j.tiles_y = (h + 63) / 64;
        j.first_tile = 0;
        pb.total_tiles = j.tiles_x * j.tiles_y;
        pb.band.band_base = p.band_base;
        pb.band.band_size = p.band_size;
        pb.band.vlt = p.vlt;
        for (int d = 0; d < kDiffs; d++) {
            pb.band.tvi[d] = p.tvi[d];
            pb.band.weight[d] = p.weight[d];
        }
        if (net->feat.count < feature_map_size(w, h)) net->feat.reset(feature_map_size(w, h));
        if (net->need.count < (size_t)pb.total_tiles + 1) net->need.reset(pb.total_tiles + 1);  // + the tile counter
        j.feat = net->feat.ptr;
        pb.need = net->need.ptr;
        pb.params = proposal_net_rounded(net, s);
        pb.frags = net->frags.ptr;
        pb.pred = pred;
        cuda_check(launch_predict(pb, s), "prediction");
    });
}

void es_proposal_net_destroy(es_proposal_net *net)
{
    if (!net) return;
    cudaDeviceSynchronize();
    delete net;
}

}  // extern "C"
