// problem.cu - upload of one DSMC problem to the device (see problem.h).
#include <cstdio>
#include <cstring>
#include <mutex>

#include "problem.h"

extern "C" {
#include "types.h"
#include "velocity.h"
}

namespace dsmc {
namespace {

// Launch-speed table of the reference model, built once on the host with the reference's
// constants (include/constants.h:17-23, src/common/velocity.c:6-47). Static, so asynchronous
// uploads from it stay valid.
const VelocityTable &speed_table() {
    static VelocityTable vt;
    static std::once_flag once;
    std::call_once(once, [] { velocity_table_init(&vt, 18e-3, 6.02e23, 1.38e-23); });
    return vt;
}

int report(char *err, size_t n, int status, const char *what, cudaError_t e) {
    if (err && n) std::snprintf(err, n, "%s: %s", what, cudaGetErrorString(e));
    return status;
}

struct Uploader {
    Problem &pr;
    cudaStream_t stream;
    bool async;
    char *err;
    size_t errlen;

    int alloc(void **p, size_t bytes) {
        const cudaError_t e = !async ? cudaMalloc(p, bytes)
                              : pr.pool ? cudaMallocFromPoolAsync(p, bytes, pr.pool, stream)
                                        : cudaMallocAsync(p, bytes, stream);
        if (e != cudaSuccess)
            return report(err, errlen, e == cudaErrorMemoryAllocation ? DSMC_ERR_NO_MEMORY : DSMC_ERR_CUDA,
                          "device allocation", e);
        pr.owned.push_back(*p);
        pr.bytes += bytes;
        return DSMC_OK;
    }

    template <typename T, typename D>
    int upload(const T *host, size_t count, D **dev) {
        static_assert(sizeof(T) == sizeof(D), "element size mismatch");
        *dev = nullptr;
        if (!host || count == 0) return DSMC_OK;
        void *p = nullptr;
        int rc = alloc(&p, count * sizeof(T));
        if (rc != DSMC_OK) return rc;
        const cudaError_t e = cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return report(err, errlen, DSMC_ERR_CUDA, "table upload", e);
        *dev = static_cast<D *>(p);
        return DSMC_OK;
    }

    template <typename T>
    int zeroed(size_t count, T **dev) {
        void *p = nullptr;
        int rc = alloc(&p, count * sizeof(T));
        if (rc != DSMC_OK) return rc;
        const cudaError_t e = cudaMemsetAsync(p, 0, count * sizeof(T), stream);
        if (e != cudaSuccess) return report(err, errlen, DSMC_ERR_CUDA, "grid clear", e);
        *dev = static_cast<T *>(p);
        return DSMC_OK;
    }
};

}  // namespace

void Problem::release() {
    for (void *q : owned) {
        if (async_alloc) cudaFreeAsync(q, stream);
        else cudaFree(q);
    }
    owned.clear();
    bytes = 0;
    t = DevTables{};
}

size_t problem_bytes(const dsmc_params *p, const dsmc_surface *s, const dsmc_collision *col) {
    const size_t ncell = static_cast<size_t>(p->hd) * p->ftd * p->ffd, nh = static_cast<size_t>(p->ftd) * p->ffd;
    size_t b = (ncell + nh) * 8;
    if (p->n_speed_bins > 0) b += ncell * p->n_speed_bins * 8;
    if (p->model == DSMC_MODEL_REFERENCE) {
        b += nh * 8 + 23 * 1000 * 8 + 23 * 4;
    } else if (s) {
        const size_t nf = static_cast<size_t>(s->nface), nn = static_cast<size_t>(20 * ((1 << (2 * s->nlevel)) - 1) / 3);
        b += nf * 9 * 8 + nf * 8 * (s->face_cdf ? 2 : 1) + 60 * 8 + nn * 9 * 8;
    }
    if (col && col->n_bg) b += static_cast<size_t>(col->n_bg_len) * 8 + ncell * (DSMC_CDF_STRIDE + 4 + 1) * 8 + ncell * 4;
    return b;
}

int problem_check(const dsmc_params *p, const dsmc_surface *s, const dsmc_collision *col,
                  char *err, size_t errlen) {
    auto bad = [&](const char *msg) {
        if (err && errlen) std::snprintf(err, errlen, "%s", msg);
        return DSMC_ERR_INVALID;
    };
    if (!p || !s) return bad("params and surface are required");
    if (p->ftd < 1 || p->ffd < 1 || p->hd < 1 || p->ftd > 4096 || p->ffd > 4096 || p->hd > 4096)
        return bad("grid dimensions out of range");
    if (!(p->dt_step > 0.0) || !(p->Radii > 0.0) || !(p->GM > 0.0) || !(p->max_height > p->Radii))
        return bad("dt, Radii, GM and max_height must be positive");
    if (p->hop_step_cap < 1) return bad("hop_step_cap must be >= 1");
    if (p->model == DSMC_MODEL_REFERENCE) {
        if (!s->T_map) return bad("reference model needs T_map");
    } else if (p->model == DSMC_MODEL_CONFIG) {
        if (!s->face_verts || !s->face_T || !s->base_centroid || !s->split_planes || s->nlevel < 0 ||
            s->nlevel > 6 || s->nface != (20 << (2 * s->nlevel)))
            return bad("config model needs a complete icosphere surface");
    } else {
        return bad("unknown model");
    }
    if (p->runner != DSMC_RUNNER_BALLISTIC && p->runner != DSMC_RUNNER_ADVANCED)
        return bad("unknown runner");
    if (col && col->n_bg &&
        (!col->cdf_coef || !col->cdf_box || !col->cdf_total || !col->cdf_valid || col->cdf_degree < 0 ||
         col->cdf_degree > DSMC_CDF_MAX_DEGREE || col->n_bg_len < 0))
        return bad("incomplete collision tables");
    if (p->n_speed_bins < 0 || p->n_speed_bins > 1024 || (p->n_speed_bins > 0 && !(p->speed_bin_width > 0.0)))
        return bad("bad speed histogram shape");
    return DSMC_OK;
}

int problem_build(Problem &pr, const dsmc_params *p, const dsmc_surface *s,
                  const dsmc_collision *col, unsigned long long *stats, cudaStream_t stream,
                  bool async_alloc, char *err, size_t errlen, cudaMemPool_t pool) {
    int rc = problem_check(p, s, col, err, errlen);
    if (rc != DSMC_OK) return rc;
    pr.release();
    pr.async_alloc = async_alloc;
    pr.stream = stream;
    pr.pool = pool;
    pr.p = *p;
    const long long ftd = p->ftd, ffd = p->ffd, hd = p->hd;
    pr.ncell = hd * ftd * ffd;
    pr.nhcell = ftd * ffd;
    pr.nhist = p->n_speed_bins > 0 ? pr.ncell * p->n_speed_bins : 0;
    Uploader u{pr, stream, async_alloc, err, errlen};
    DevTables &t = pr.t;
    t = DevTables{};
    if (p->model == DSMC_MODEL_REFERENCE) {
        const VelocityTable &vt = speed_table();
        const double *d_T = nullptr, *d_sp = nullptr;
        const int *d_cnt = nullptr;
        if ((rc = u.upload(s->T_map, static_cast<size_t>(ftd * ffd), &d_T)) != DSMC_OK) return rc;
        if ((rc = u.upload(&vt.speeds[0][0], 23 * 1000, &d_sp)) != DSMC_OK) return rc;
        if ((rc = u.upload(vt.count, 23, &d_cnt)) != DSMC_OK) return rc;
        t.T_map = d_T;
        t.vt_speeds = d_sp;
        t.vt_count = d_cnt;
    } else {
        const size_t nf = static_cast<size_t>(s->nface);
        const size_t nnode = static_cast<size_t>(20 * ((1 << (2 * s->nlevel)) - 1) / 3);
        t.nface = s->nface;
        t.nlevel = s->nlevel;
        const double *dv = nullptr, *dT = nullptr, *dc = nullptr, *db = nullptr, *dp = nullptr;
        if ((rc = u.upload(s->face_verts, nf * 9, &dv)) != DSMC_OK) return rc;
        if ((rc = u.upload(s->face_T, nf, &dT)) != DSMC_OK) return rc;
        if ((rc = u.upload(s->face_cdf, nf, &dc)) != DSMC_OK) return rc;
        if ((rc = u.upload(s->base_centroid, static_cast<size_t>(60), &db)) != DSMC_OK) return rc;
        if ((rc = u.upload(s->split_planes, nnode * 9, &dp)) != DSMC_OK) return rc;
        t.face_verts = dv;
        t.face_T = dT;
        t.face_cdf = dc;
        t.base_centroid = db;
        t.split_planes = dp;
    }
    if (col && col->n_bg) {
        const size_t nc = static_cast<size_t>(pr.ncell);
        const double *nb = nullptr, *cc = nullptr, *cb = nullptr, *ct = nullptr;
        const int *cv = nullptr;
        if ((rc = u.upload(col->n_bg, static_cast<size_t>(col->n_bg_len), &nb)) != DSMC_OK) return rc;
        if ((rc = u.upload(col->cdf_coef, nc * DSMC_CDF_STRIDE, &cc)) != DSMC_OK) return rc;
        if ((rc = u.upload(col->cdf_box, nc * 4, &cb)) != DSMC_OK) return rc;
        if ((rc = u.upload(col->cdf_total, nc, &ct)) != DSMC_OK) return rc;
        if ((rc = u.upload(reinterpret_cast<const int *>(col->cdf_valid), nc, &cv)) != DSMC_OK) return rc;
        t.n_bg = nb;
        t.n_bg_len = col->n_bg_len;
        t.cdf_coef = cc;
        t.cdf_box = cb;
        t.cdf_total = ct;
        t.cdf_valid = cv;
        t.cdf_degree = col->cdf_degree;
    }
    if ((rc = u.zeroed(static_cast<size_t>(pr.ncell), &t.density)) != DSMC_OK) return rc;
    if ((rc = u.zeroed(static_cast<size_t>(pr.nhcell), &t.horizon)) != DSMC_OK) return rc;
    if (pr.nhist > 0 && (rc = u.zeroed(static_cast<size_t>(pr.nhist), &t.speed_hist)) != DSMC_OK) return rc;
    t.stats = stats;
    // the host arrays of the caller are pageable: the copies above have been staged when the
    // calls returned, but wait for the device so that errors surface here
    const cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return report(err, errlen, DSMC_ERR_CUDA, "problem upload", e);
    return DSMC_OK;
}

}  // namespace dsmc
