// C ABI of the learned SGS closure (mlp.cu): create / train / evaluate / save.
// No counterpart in the reference (it stands in for VremanSGS / DSMSGS).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "mc3d_internal.h"

using namespace mc3d;

struct mc3d_mlp_s {
    MlpDev dev;
    int device = 0;
    // training workspace, sized for the largest batch seen
    int cap = 0;
    float *act = nullptr, *out = nullptr, *delta = nullptr;
    double *loss = nullptr;
};

namespace {

int mlp_alloc_ws(mc3d_mlp m, int n) {
    if (n <= m->cap) return MC3D_OK;
    cudaFree(m->act);
    cudaFree(m->out);
    cudaFree(m->delta);
    m->act = m->out = m->delta = nullptr;
    m->cap = 0;
    MC3D_CUDA_TRY(cudaMalloc(&m->act, (size_t)6 * n * 64 * sizeof(float)));
    MC3D_CUDA_TRY(cudaMalloc(&m->out, (size_t)n * MLP_OUT * sizeof(float)));
    MC3D_CUDA_TRY(cudaMalloc(&m->delta, ((size_t)3 * n * 64 + (size_t)n * MLP_OUT) * sizeof(float)));
    m->cap = n;
    return MC3D_OK;
}

const char MAGIC[8] = {'M', 'C', '3', 'D', 'M', 'L', 'P', '1'};

}  // namespace

extern "C" {

int mc3d_mlp_create(unsigned long long seed, int device, mc3d_mlp *out) {
    if (!out) return fail(MC3D_ERR_ARG, "null argument");
    *out = nullptr;
    MC3D_CUDA_TRY(cudaSetDevice(device));
    mc3d_mlp m = new mc3d_mlp_s();
    m->device = device;
    // Xavier-uniform weights, zero biases
    std::vector<float> P(MLP_NPARAM, 0.0f);
    std::mt19937_64 rng(seed);
    const int fan[4][2] = {{MLP_IN, 64}, {64, 64}, {64, 64}, {64, MLP_OUT}};
    int off = 0;
    for (int l = 0; l < 4; l++) {
        const int nin = fan[l][0], nout = fan[l][1];
        const double a = std::sqrt(6.0 / (nin + nout));
        std::uniform_real_distribution<double> U(-a, a);
        for (int k = 0; k < nin * nout; k++) P[off + k] = (float)U(rng);
        off += nin * nout + nout;
    }
    for (int k = 0; k < MLP_IN; k++) {
        m->dev.norm.mean[k] = 0.0f;
        m->dev.norm.inv_std[k] = 1.0f;
        m->dev.norm.lo[k] = -INFINITY;
        m->dev.norm.hi[k] = INFINITY;
    }
    for (int k = 0; k < MLP_OUT; k++) {
        m->dev.norm.ymean[k] = 0.0f;
        m->dev.norm.ystd[k] = 1.0f;
    }
    cudaError_t e = cudaSuccess;
    float **bufs[4] = {&m->dev.P, &m->dev.G, &m->dev.M, &m->dev.V};
    for (float **b : bufs) {
        if (e == cudaSuccess) e = cudaMalloc(b, MLP_NPARAM * sizeof(float));
        if (e == cudaSuccess) e = cudaMemset(*b, 0, MLP_NPARAM * sizeof(float));
    }
    if (e == cudaSuccess) e = cudaMalloc(&m->dev.Tw, MLPT_BYTES);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(m->dev.P, P.data(), MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        mc3d_mlp_destroy(m);
        return fail(MC3D_ERR_CUDA, std::string("mc3d_mlp_create: ") + cudaGetErrorString(e));
    }
    int rc = mlp_pack(m->dev, nullptr);
    if (rc) {
        mc3d_mlp_destroy(m);
        return rc;
    }
    MC3D_CUDA_TRY(cudaDeviceSynchronize());
    *out = m;
    return MC3D_OK;
}

int mc3d_mlp_destroy(mc3d_mlp m) {
    if (!m) return MC3D_OK;
    cudaSetDevice(m->device);
    for (void *p : {(void *)m->dev.P, (void *)m->dev.G, (void *)m->dev.M, (void *)m->dev.V, (void *)m->dev.Tw,
                    (void *)m->act, (void *)m->out, (void *)m->delta, (void *)m->loss})
        if (p) cudaFree(p);
    delete m;
    return MC3D_OK;
}

int mc3d_mlp_set_normalization(mc3d_mlp m, const float *mean, const float *std, const float *lo, const float *hi,
                               const float *ymean, const float *ystd) {
    if (!m || !mean || !std || !lo || !hi || !ymean || !ystd) return fail(MC3D_ERR_ARG, "null argument");
    for (int k = 0; k < MLP_IN; k++) {
        if (!(std[k] > 0)) return fail(MC3D_ERR_ARG, "feature standard deviations must be positive");
        m->dev.norm.mean[k] = mean[k];
        m->dev.norm.inv_std[k] = 1.0f / std[k];
        m->dev.norm.lo[k] = lo[k];
        m->dev.norm.hi[k] = hi[k];
    }
    for (int k = 0; k < MLP_OUT; k++) {
        if (!(ystd[k] > 0)) return fail(MC3D_ERR_ARG, "target standard deviations must be positive");
        m->dev.norm.ymean[k] = ymean[k];
        m->dev.norm.ystd[k] = ystd[k];
    }
    return MC3D_OK;
}

int mc3d_mlp_get_normalization(mc3d_mlp m, float *out /* 4*9 + 2*2 */) {
    if (!m || !out) return fail(MC3D_ERR_ARG, "null argument");
    for (int k = 0; k < MLP_IN; k++) {
        out[k] = m->dev.norm.mean[k];
        out[MLP_IN + k] = 1.0f / m->dev.norm.inv_std[k];
        out[2 * MLP_IN + k] = m->dev.norm.lo[k];
        out[3 * MLP_IN + k] = m->dev.norm.hi[k];
    }
    for (int k = 0; k < MLP_OUT; k++) {
        out[4 * MLP_IN + k] = m->dev.norm.ymean[k];
        out[4 * MLP_IN + MLP_OUT + k] = m->dev.norm.ystd[k];
    }
    return MC3D_OK;
}

int mc3d_mlp_train_step(mc3d_mlp m, const float *x, const float *y, int n, float lr, double *loss, void *stream) {
    if (!m || !x || !y || n <= 0) return fail(MC3D_ERR_ARG, "bad argument");
    MC3D_CUDA_TRY(cudaSetDevice(m->device));
    int rc = mlp_alloc_ws(m, n);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    MC3D_CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(double), st));
    if ((rc = mlp_train_step(m->dev, x, y, n, lr, m->act, m->out, m->delta, m->loss, st))) return rc;
    if (loss) {
        MC3D_CUDA_TRY(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        MC3D_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return MC3D_OK;
}

int mc3d_mlp_gradient(mc3d_mlp m, const float *x, const float *y, int n, float *G, double *loss, void *stream) {
    if (!m || !x || !y || !G || n <= 0) return fail(MC3D_ERR_ARG, "bad argument");
    MC3D_CUDA_TRY(cudaSetDevice(m->device));
    int rc = mlp_alloc_ws(m, n);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    MC3D_CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(double), st));
    MC3D_CUDA_TRY(cudaMemsetAsync(m->dev.G, 0, MLP_NPARAM * sizeof(float), st));
    if ((rc = mlp_gradient(m->dev, x, y, n, m->act, m->out, m->delta, m->loss, st))) return rc;
    MC3D_CUDA_TRY(cudaMemcpyAsync(G, m->dev.G, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (loss) MC3D_CUDA_TRY(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    // the training step expects a zero gradient buffer
    MC3D_CUDA_TRY(cudaMemsetAsync(m->dev.G, 0, MLP_NPARAM * sizeof(float), st));
    MC3D_CUDA_TRY(cudaStreamSynchronize(st));
    return MC3D_OK;
}

int mc3d_mlp_forward(mc3d_mlp m, const float *x, float *y, int n, void *stream) {
    if (!m || !x || !y || n <= 0) return fail(MC3D_ERR_ARG, "bad argument");
    MC3D_CUDA_TRY(cudaSetDevice(m->device));
    return mlp_forward_fp32(m->dev, x, n, nullptr, y, (cudaStream_t)stream);
}

int mc3d_mlp_infer_bf16(mc3d_mlp m, const float *x, float *y, int n, void *stream) {
    if (!m || !x || !y || n <= 0) return fail(MC3D_ERR_ARG, "bad argument");
    MC3D_CUDA_TRY(cudaSetDevice(m->device));
    return mlp_infer_bf16(m->dev, x, n, y, (cudaStream_t)stream);
}

int mc3d_mlp_get_params(mc3d_mlp m, float *P) {
    if (!m || !P) return fail(MC3D_ERR_ARG, "null argument");
    MC3D_CUDA_TRY(cudaSetDevice(m->device));
    MC3D_CUDA_TRY(cudaDeviceSynchronize());
    MC3D_CUDA_TRY(cudaMemcpy(P, m->dev.P, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return MC3D_OK;
}

int mc3d_mlp_set_params(mc3d_mlp m, const float *P) {
    if (!m || !P) return fail(MC3D_ERR_ARG, "null argument");
    MC3D_CUDA_TRY(cudaSetDevice(m->device));
    MC3D_CUDA_TRY(cudaMemcpy(m->dev.P, P, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    int rc = mlp_pack(m->dev, nullptr);
    if (rc) return rc;
    MC3D_CUDA_TRY(cudaDeviceSynchronize());
    return MC3D_OK;
}

// file: 8-byte magic, the normalisation (4*9 + 2*2 floats), the 9090 parameters
int mc3d_mlp_save(mc3d_mlp m, const char *path) {
    if (!m || !path) return fail(MC3D_ERR_ARG, "null argument");
    std::vector<float> P(MLP_NPARAM), nrm(4 * MLP_IN + 2 * MLP_OUT);
    int rc = mc3d_mlp_get_params(m, P.data());
    if (rc) return rc;
    mc3d_mlp_get_normalization(m, nrm.data());
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(MC3D_ERR_ARG, std::string("cannot write ") + path);
    bool ok = std::fwrite(MAGIC, 1, 8, f) == 8 && std::fwrite(nrm.data(), sizeof(float), nrm.size(), f) == nrm.size() &&
              std::fwrite(P.data(), sizeof(float), P.size(), f) == P.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? MC3D_OK : fail(MC3D_ERR_ARG, std::string("short write to ") + path);
}

int mc3d_mlp_load(mc3d_mlp m, const char *path) {
    if (!m || !path) return fail(MC3D_ERR_ARG, "null argument");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(MC3D_ERR_ARG, std::string("cannot read ") + path);
    char mg[8];
    std::vector<float> P(MLP_NPARAM), nrm(4 * MLP_IN + 2 * MLP_OUT);
    bool ok = std::fread(mg, 1, 8, f) == 8 && std::memcmp(mg, MAGIC, 8) == 0 &&
              std::fread(nrm.data(), sizeof(float), nrm.size(), f) == nrm.size() &&
              std::fread(P.data(), sizeof(float), P.size(), f) == P.size();
    std::fclose(f);
    if (!ok) return fail(MC3D_ERR_ARG, std::string("not an MLP closure file: ") + path);
    int rc = mc3d_mlp_set_normalization(m, nrm.data(), nrm.data() + MLP_IN, nrm.data() + 2 * MLP_IN,
                                        nrm.data() + 3 * MLP_IN, nrm.data() + 4 * MLP_IN,
                                        nrm.data() + 4 * MLP_IN + MLP_OUT);
    if (rc) return rc;
    return mc3d_mlp_set_params(m, P.data());
}

int mc3d_sgs_box_filter(const double *const q[5], int Nx, int Ny, int Nz, int f, double *const out[14],
                        void *stream) {
    if (!q || !out || f <= 0 || Nx % f || Ny % f || Nz % f) return fail(MC3D_ERR_ARG, "bad box filter arguments");
    return launch_box_filter(Grid3{Nx, Ny, Nz}, f, q, out, (cudaStream_t)stream);
}

int mc3d_sgs_training_pairs(const double *const coarse[14], const double *const grads[12], int Nx, int Ny, int Nz,
                            const double jd[3], double delta, double mu_ref, float *x, float *y, void *stream) {
    if (!coarse || !grads || !jd || !x || !y) return fail(MC3D_ERR_ARG, "null argument");
    return launch_training_pairs(Grid3{Nx, Ny, Nz}, coarse, grads, jd, delta, mu_ref, x, y, (cudaStream_t)stream);
}

}  // extern "C"

namespace mc3d {
const MlpDev *mlp_dev(mc3d_mlp m) { return m ? &m->dev : nullptr; }
}  // namespace mc3d
