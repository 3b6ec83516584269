/*
 * kelp_oracle.c -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * A plain-C CPU restatement of KELP's compiled time-stepping path, used as the
 * parity checker for the CUDA kernels (tests/, __graft_entry__.smoke()) and as
 * the timed CPU baseline of bench.py.  Nothing in kelp_b200/ links or calls it.
 *
 * It works on the reference's own array layout (dense node_to_elems (N,
 * max_conn), elem_nodes (E, max_v), node_xyz (N, 3), CSR grid hash) and follows
 * the reference's Numba functions statement by statement, with the C
 * library's math (the functions Numba lowers np.cos/np.sin/math.log to) and no
 * floating-point contraction (-ffp-contract=off).  Each function cites the
 * reference file:line it restates (paths inside the KELP project).
 *
 * Pinned against golden vectors produced by running the reference itself
 * (tests/golden/make_golden.py -> tests/golden/*.npz; tests/test_oracle_golden.py).
 */
#include <math.h>
#include <pthread.h>
#include <unistd.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DEG2RAD 0.017453292519943295
#define RAD2DEG 57.29577951308232
#define SLM 111120.0
#define R_STD 6371000.0
#define BARY_EPS (-1e-6)
#define AREA_TOL 1e-10
#define ALIVE 1
#define OUTSIDE 3
#define NOT_RELEASED 4

typedef struct {
    int64_t N, E;
    int max_v, max_conn;
    const double *lon, *lat, *depth, *xyz, *zlev;
    const int32_t *en, *n2e, *n2e_cnt, *gh_off, *gh_ids;
    double cell, lon_min, lat_min, r_earth;
    int nx, ny, wrap, far_rows, exact, K;
    const double *dl_p, *dl_bed;      /* depth-linear table (vertical_uv.py:181-278) */
    const int32_t* dl_last;
    int dl_M;
    const int32_t* enb;   /* (E, max_v) edge neighbours of the compacted ring (walk), or NULL */
    const double* sigma;  /* (K) sigma interfaces, 1 surface -> 0 bed (vertical_coord "sigma"), or NULL */
    int sig;
    int cg;                        /* 1: a NEMO C-grid mesh (readers/nemo/_mesh.py build_nemo_cgrid_mesh) */
    const int32_t* cg_corners;     /* (E, 4) F-point corners SW, SE, NE, NW */
    const int64_t* cg_ji;          /* (E, 2) T-cell (j, i) */
    const int32_t* cg_nlev;        /* (E) wet levels (0: the dry ring) */
    const int32_t* cg_nlev_r;      /* (ny*nx) wet levels per column */
    int cg_nx, cg_K, cg_shrunk, cg_has_e;
    int64_t cg_nynx;
    const double *cg_e2u, *cg_e1v, *cg_area, *cg_zw, *cg_e3b, *cg_e3u, *cg_e3v;
    const int32_t *cg_kbu, *cg_kbv;
    const double *ec_lon, *ec_lat;   /* (E) element centres (least-squares u/v), or NULL */
} OMesh;

typedef struct {
    const void *ua, *va, *wa, *ub, *vb, *wb, *ut, *vt, *wt;
    int f32;
    double alpha0;
    int64_t n;
    const void *aza, *azb;   /* vertical diffusivity (K, N) of the bracket pair, or NULL */
    const double *etaa, *etab, *etat;   /* free surface (N) of the pair and target (sigma meshes) */
    int pchip;                          /* 1: a, b, t, d are a PCHIP stencil at times pt; alphas are times */
    const void *ud, *vd, *wd;
    const double* etad;
    double pt[4];
    int lsq;                            /* 1: 2-D u/v on element centres by least squares (n = E) */
} OField;

static double fld(const void* p, int f32, int64_t i) {
    return f32 ? (double)((const float*)p)[i] : ((const double*)p)[i];
}

/* Python float % for a positive divisor (CPython float_rem). */
static double pymod(double x, double m) {
    double r = fmod(x, m);
    if (r != 0.0) {
        if (r < 0.0) r += m;
    } else {
        r = 0.0;
    }
    return r;
}
static double wrap180(double x) { return pymod(x + 180.0, 360.0) - 180.0; }
static int imod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

/* mesh.py:1192-1207 */
static double fold_dlon(const OMesh* m, double lon_p) {
    double dlon = pymod(lon_p - m->lon_min, 360.0);
    if (!m->wrap) {
        double grid_span = m->nx * m->cell;
        if (dlon > grid_span && (dlon - grid_span) > (360.0 - dlon)) dlon -= 360.0;
    }
    return dlon;
}

/* mesh.py:1210-1232 */
static void cell_of(const OMesh* m, double lon_p, double lat_p, int* ci, int* cj) {
    double dlon = fold_dlon(m, lon_p);
    int a = (int)(dlon / m->cell);
    int b = (int)((lat_p - m->lat_min) / m->cell);
    if (a < 0) a = 0;
    if (a >= m->nx) a = m->nx - 1;
    if (b < 0) b = 0;
    if (b >= m->ny) b = m->ny - 1;
    *ci = a;
    *cj = b;
}

static void qxyz(double lon_p, double lat_p, double* xp, double* yp, double* zp, double* cl) {
    double lat_r = lat_p * DEG2RAD, lon_r = lon_p * DEG2RAD;
    double c = cos(lat_r);
    *xp = c * cos(lon_r);
    *yp = c * sin(lon_r);
    *zp = sin(lat_r);
    *cl = c;
}

static void scan_cell(const OMesh* m, int cell, double xp, double yp, double zp, int* best, double* bd2) {
    for (int k = m->gh_off[cell]; k < m->gh_off[cell + 1]; ++k) {
        int n = m->gh_ids[k];
        double xn = m->xyz[3 * (int64_t)n], yn = m->xyz[3 * (int64_t)n + 1], zn = m->xyz[3 * (int64_t)n + 2];
        double d2 = (xn - xp) * (xn - xp) + (yn - yp) * (yn - yp) + (zn - zp) * (zn - zp);
        if (d2 < *bd2) { *bd2 = d2; *best = n; }
    }
}

static void scan_row_range(const OMesh* m, int cj2, int lo, int hi, double xp, double yp, double zp, int* best, double* bd2) {
    for (int k = m->gh_off[cj2 * m->nx + lo]; k < m->gh_off[cj2 * m->nx + hi + 1]; ++k) {
        int n = m->gh_ids[k];
        double xn = m->xyz[3 * (int64_t)n], yn = m->xyz[3 * (int64_t)n + 1], zn = m->xyz[3 * (int64_t)n + 2];
        double d2 = (xn - xp) * (xn - xp) + (yn - yp) * (yn - yp) + (zn - zp) * (zn - zp);
        if (d2 < *bd2) { *bd2 = d2; *best = n; }
    }
}

/* mesh.py:1235-1303 */
static int nearest_3x3(const OMesh* m, double lon_p, double lat_p) {
    int ci, cj;
    cell_of(m, lon_p, lat_p, &ci, &cj);
    double xp, yp, zp, cl;
    qxyz(lon_p, lat_p, &xp, &yp, &zp, &cl);
    int best = -1;
    double bd2 = 1e30;
    for (int dj = -1; dj <= 1; ++dj) {
        int cj2 = cj + dj;
        if (cj2 < 0 || cj2 >= m->ny) continue;
        for (int di = -1; di <= 1; ++di) {
            int ci2 = ci + di;
            if (ci2 < 0) ci2 = m->wrap ? ci2 + m->nx : -1;
            else if (ci2 >= m->nx) ci2 = m->wrap ? ci2 - m->nx : -1;
            if (ci2 < 0) continue;
            scan_cell(m, cj2 * m->nx + ci2, xp, yp, zp, &best, &bd2);
        }
    }
    return best;
}

/* mesh.py:1306-1328 */
static void cap_extents(double lon_p, double lat_p, double lon_n, double lat_n, double* th, double* ext) {
    double lat_pr = lat_p * DEG2RAD, lat_nr = lat_n * DEG2RAD;
    double cosd = sin(lat_pr) * sin(lat_nr) + cos(lat_pr) * cos(lat_nr) * cos((lon_p - lon_n) * DEG2RAD);
    if (cosd > 1.0) cosd = 1.0;
    if (cosd < -1.0) cosd = -1.0;
    double theta = acos(cosd);
    if (theta <= 0.0) { *th = 0.0; *ext = 0.0; return; }
    *th = theta * RAD2DEG;
    if (fabs(lat_p) + *th >= 90.0) { *ext = 1.0e30; return; }
    double r = sin(theta) / cos(lat_pr);
    if (r >= 1.0) { *ext = 1.0e30; return; }
    *ext = asin(r) * RAD2DEG;
}

/* mesh.py:1475-1549 */
static int provable_rect(const OMesh* m, double lon_p, double lat_p, int node, int rx, int ry) {
    double th, ext;
    cap_extents(lon_p, lat_p, m->lon[node], m->lat[node], &th, &ext);
    if (th <= 0.0) return 0;
    double dlon = fold_dlon(m, lon_p);
    double lon_q = m->lon_min + dlon;
    int ci_raw = (int)floor(dlon / m->cell);
    int cj_raw = (int)floor((lat_p - m->lat_min) / m->cell);
    double INF = 1.0e30;
    int cj = cj_raw;
    if (cj < 0) cj = 0;
    if (cj > m->ny - 1) cj = m->ny - 1;
    double cov_dn = cj - ry >= 0 ? lat_p - (m->lat_min + (cj - ry) * m->cell) : INF;
    double cov_up = cj + ry <= m->ny - 1 ? (m->lat_min + (cj + ry + 1) * m->cell) - lat_p : INF;
    int code = 0;
    if (th > cov_dn || th > cov_up) code |= 1;
    if (m->wrap) {
        if (2 * rx + 1 >= m->nx) return code;
        if (ext >= INF) return code | 4;
        double w_last = 360.0 - (m->nx - 1) * m->cell;
        int ci = imod(ci_raw, m->nx);
        double left = m->lon_min + (ci - rx) * m->cell;
        if (ci - rx < 0) left += m->cell - w_last;
        double right = m->lon_min + (ci + rx + 1) * m->cell;
        if (ci + rx >= m->nx - 1) right -= m->cell - w_last;
        if (ext > lon_q - left || ext > right - lon_q) code |= 2;
        return code;
    }
    int ci = ci_raw;
    if (ci < 0) ci = 0;
    if (ci > m->nx - 1) ci = m->nx - 1;
    double cov_l = ci - rx >= 0 ? lon_q - (m->lon_min + (ci - rx) * m->cell) : INF;
    double cov_r = ci + rx <= m->nx - 1 ? (m->lon_min + (ci + rx + 1) * m->cell) - lon_q : INF;
    if (cov_l >= INF && cov_r >= INF) return code;
    if (ext >= INF) return code | 4;
    if (ext > cov_l || ext > cov_r) code |= 2;
    double n_lo = m->lon_min + m->cell, n_hi = m->lon_min + (m->nx - 1) * m->cell;
    double shifts[2] = {-360.0, 360.0};
    for (int s = 0; s < 2; ++s) {
        double a = lon_q - ext + shifts[s], b = lon_q + ext + shifts[s];
        if (b >= n_lo && a <= n_hi) return code | 4;
    }
    return code;
}

/* mesh.py:1331-1442 */
static int nearest_widened(const OMesh* m, double lon_p, double lat_p) {
    int best = nearest_3x3(m, lon_p, lat_p);
    if (best >= 0) return best;
    int ci, cj;
    cell_of(m, lon_p, lat_p, &ci, &cj);
    double xp, yp, zp, cl;
    qxyz(lon_p, lat_p, &xp, &yp, &zp, &cl);
    double bd2 = 1e30;
    int max_ring = m->nx > m->ny ? m->nx : m->ny;
    int found = -1;
    for (int r = 2; r <= max_ring; ++r) {
        for (int dj = -r; dj <= r; ++dj) {
            int cj2 = cj + dj;
            if (cj2 < 0 || cj2 >= m->ny) continue;
            int step = (dj == -r || dj == r) ? 1 : 2 * r;
            for (int di = -r; di <= r; di += step) {
                int ci2 = ci + di;
                if (m->wrap) ci2 = imod(ci2, m->nx);
                else if (ci2 < 0 || ci2 >= m->nx) continue;
                scan_cell(m, cj2 * m->nx + ci2, xp, yp, zp, &best, &bd2);
            }
        }
        if (best >= 0) {
            if (found < 0) found = r;
            else if (r > found) break;
        }
    }
    return best;
}

static void scan_row_window(const OMesh* m, int cj2, int ci, int rx, double xp, double yp, double zp, int* best, double* bd2) {
    if (m->wrap && 2 * rx + 1 >= m->nx) { scan_row_range(m, cj2, 0, m->nx - 1, xp, yp, zp, best, bd2); return; }
    int lo = ci - rx, hi = ci + rx;
    if (m->wrap) {
        if (lo < 0) { scan_row_range(m, cj2, lo + m->nx, m->nx - 1, xp, yp, zp, best, bd2); lo = 0; }
        else if (hi > m->nx - 1) { scan_row_range(m, cj2, 0, hi - m->nx, xp, yp, zp, best, bd2); hi = m->nx - 1; }
    } else {
        if (lo < 0) lo = 0;
        if (hi > m->nx - 1) hi = m->nx - 1;
    }
    scan_row_range(m, cj2, lo, hi, xp, yp, zp, best, bd2);
}

/* mesh.py:1611-1859 */
static int nearest_exact(const OMesh* m, double lon_p, double lat_p) {
    double far = m->far_rows * m->cell;
    if (lat_p < m->lat_min - far || lat_p > m->lat_min + m->ny * m->cell + far)
        return nearest_widened(m, lon_p, lat_p);
    int best = nearest_3x3(m, lon_p, lat_p);
    int code = 0;
    if (best >= 0) {
        code = provable_rect(m, lon_p, lat_p, best, 1, 1);
        if (code == 0) return best;
        double th, ext;
        cap_extents(lon_p, lat_p, m->lon[best], m->lat[best], &th, &ext);
        if (th > far) return best;
    }
    int ci, cj;
    cell_of(m, lon_p, lat_p, &ci, &cj);
    double xp, yp, zp, cos_lat_p;
    qxyz(lon_p, lat_p, &xp, &yp, &zp, &cos_lat_p);
    double best_d2 = 1.0e30;
    if (best >= 0) {
        double xn = m->xyz[3 * (int64_t)best], yn = m->xyz[3 * (int64_t)best + 1], zn = m->xyz[3 * (int64_t)best + 2];
        best_d2 = (xn - xp) * (xn - xp) + (yn - yp) * (yn - yp) + (zn - zp) * (zn - zp);
    }
    int rx = 1, ry = 1;
    int short_row = 360.0 * cos_lat_p <= 32 * m->cell;
    int rx_max;
    if (m->wrap) { rx_max = m->nx / 2; if (rx_max < 1) rx_max = 1; }
    else rx_max = ci > m->nx - 1 - ci ? ci : m->nx - 1 - ci;
    int ry_max = cj > m->ny - 1 - cj ? cj : m->ny - 1 - cj;
    double abs_lat = lat_p >= 0.0 ? lat_p : -lat_p;
    double dlon_q = fold_dlon(m, lon_p);
    double INF = 1.0e30;
    for (;;) {
        if (best >= 0 && code == 0) {
            code = provable_rect(m, lon_p, lat_p, best, rx, ry);
            if (code == 0) return best;
        }
        if (best < 0 || 2.0 * asin(0.5 * sqrt(best_d2)) * RAD2DEG > far) {
            int cols_full = m->wrap ? (2 * rx + 1 >= m->nx) : (ci - rx <= 0 && ci + rx >= m->nx - 1);
            double clear = ry >= ry_max ? INF : ry * m->cell;
            if (!cols_full) {
                double lat_edge = abs_lat + (ry + 1) * m->cell;
                double clear_lon;
                if (lat_edge >= 90.0) clear_lon = 0.0;
                else {
                    double dl = rx * m->cell;
                    if (!m->wrap) {
                        double x = dlon_q > 0.0 ? dlon_q : 0.0;
                        double w = m->nx * m->cell;
                        if (x > w) x = w;
                        double near_edge = x < w - x ? x : w - x;
                        double dl_cut = 360.0 - w + near_edge;
                        if (dl_cut < dl) dl = dl_cut;
                    }
                    if (dl > 180.0) dl = 180.0;
                    clear_lon = asin(sin(dl * DEG2RAD) * cos(lat_edge * DEG2RAD)) * RAD2DEG;
                }
                if (clear_lon < clear) clear = clear_lon;
            }
            if (clear >= far) {
                if (best >= 0) return best;
                return nearest_widened(m, lon_p, lat_p);
            }
        }
        int gx, gy, ax;
        if (best >= 0) { gx = (code & 2) != 0; gy = (code & 1) != 0; ax = (code & 4) != 0; code = 0; }
        else if (short_row) { gx = 0; gy = 1; ax = 1; }
        else { gx = 1; gy = 1; ax = 0; }
        if (rx >= rx_max) { gx = 0; ax = 0; }
        if (ry >= ry_max) gy = 0;
        if (!(gx || gy || ax)) {
            if (best >= 0) return best;
            return nearest_widened(m, lon_p, lat_p);
        }
        int rx_new = ax ? rx_max : (gx ? rx + 1 : rx);
        int ry_new = gy ? ry + 1 : ry;
        int j_lo = cj - ry > 0 ? cj - ry : 0;
        int j_hi = cj + ry < m->ny - 1 ? cj + ry : m->ny - 1;
        if (rx_new > rx) {
            if (m->wrap && 2 * rx_new + 1 >= m->nx && rx_new - rx > 1) {
                for (int cj2 = j_lo; cj2 <= j_hi; ++cj2) {
                    int lo = imod(ci + rx + 1, m->nx), hi = imod(ci - rx - 1, m->nx);
                    if (lo <= hi) scan_row_range(m, cj2, lo, hi, xp, yp, zp, &best, &best_d2);
                    else {
                        scan_row_range(m, cj2, lo, m->nx - 1, xp, yp, zp, &best, &best_d2);
                        scan_row_range(m, cj2, 0, hi, xp, yp, zp, &best, &best_d2);
                    }
                }
            } else if (!m->wrap && rx_new - rx > 1) {
                for (int cj2 = j_lo; cj2 <= j_hi; ++cj2) {
                    if (ci - rx - 1 >= 0) {
                        int lo = ci - rx_new > 0 ? ci - rx_new : 0;
                        scan_row_range(m, cj2, lo, ci - rx - 1, xp, yp, zp, &best, &best_d2);
                    }
                    if (ci + rx + 1 <= m->nx - 1) {
                        int hi = ci + rx_new < m->nx - 1 ? ci + rx_new : m->nx - 1;
                        scan_row_range(m, cj2, ci + rx + 1, hi, xp, yp, zp, &best, &best_d2);
                    }
                }
            } else {
                for (int r = rx + 1; r <= rx_new; ++r) {
                    if (m->wrap) {
                        int cl2 = imod(ci - r, m->nx), cr2 = imod(ci + r, m->nx);
                        int two = 2 * r + 1 <= m->nx;
                        for (int cj2 = j_lo; cj2 <= j_hi; ++cj2) {
                            scan_cell(m, cj2 * m->nx + cl2, xp, yp, zp, &best, &best_d2);
                            if (two) scan_cell(m, cj2 * m->nx + cr2, xp, yp, zp, &best, &best_d2);
                        }
                    } else {
                        int cs[2] = {ci - r, ci + r};
                        for (int s = 0; s < 2; ++s) {
                            if (cs[s] < 0 || cs[s] > m->nx - 1) continue;
                            for (int cj2 = j_lo; cj2 <= j_hi; ++cj2)
                                scan_cell(m, cj2 * m->nx + cs[s], xp, yp, zp, &best, &best_d2);
                        }
                    }
                }
            }
        }
        for (int r = ry + 1; r <= ry_new; ++r) {
            int rows[2] = {cj - r, cj + r};
            for (int s = 0; s < 2; ++s) {
                if (rows[s] < 0 || rows[s] > m->ny - 1) continue;
                scan_row_window(m, rows[s], ci, rx_new, xp, yp, zp, &best, &best_d2);
            }
        }
        rx = rx_new;
        ry = ry_new;
    }
}

/* integrators.py:1470-1487 */
static int anchor(const OMesh* m, double lon_p, double lat_p) {
    return m->exact ? nearest_exact(m, lon_p, lat_p) : nearest_widened(m, lon_p, lat_p);
}

/* mesh.py:2054-2073 */
static void bary_tri(double px, double py, const double* tx, const double* ty, double* w) {
    double ax = tx[0], ay = ty[0], bx = tx[1], by = ty[1], cx = tx[2], cy = ty[2];
    double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
    if (fabs(denom) < AREA_TOL) { w[0] = w[1] = w[2] = -1.0; return; }
    w[0] = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
    w[1] = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
    w[2] = 1.0 - w[0] - w[1];
}

/* mesh.py:2076-2116 */
static void wachspress(double px, double py, const double* x, const double* y, double* out) {
    double A[4], Cc[4], s = 0.0;
    for (int k = 0; k < 4; ++k) {
        int i1 = (k + 1) % 4, im = (k + 3) % 4;
        A[k] = (x[k] - px) * (y[i1] - py) - (x[i1] - px) * (y[k] - py);
        Cc[k] = (x[k] - x[im]) * (y[i1] - y[im]) - (x[i1] - x[im]) * (y[k] - y[im]);
    }
    for (int k = 0; k < 4; ++k) { out[k] = Cc[k] * A[(k + 1) % 4] * A[(k + 2) % 4]; s += out[k]; }
    for (int k = 0; k < 4; ++k) out[k] = out[k] / s;
}

/* mesh.py:2119-2136 */
static void polygon_weights(double px, double py, const double* x, const double* y, int nv, double* w) {
    if (nv == 3) {
        double t[3];
        bary_tri(px, py, x, y, t);
        w[0] = t[0]; w[1] = t[1]; w[2] = t[2];
        return;
    }
    wachspress(px, py, x, y, w);
}

/* mesh.py:2210-2263 + :2006-2051 + :2139-2168 */
static int element_contains(const OMesh* m, int c, double lon_p, double lat_p) {
    const int32_t* nodes = m->en + (int64_t)c * m->max_v;
    int mask[4] = {0, 0, 0, 0};
    for (int k = 0; k < m->max_v; ++k) mask[k] = nodes[k] >= 0;
    if (m->max_v == 4 && nodes[3] == nodes[0] && nodes[0] >= 0) mask[3] = 0;
    double ln[4], la[4];
    int n = 0;
    for (int k = 0; k < m->max_v; ++k)
        if (mask[k]) { ln[n] = m->lon[nodes[k]]; la[n] = m->lat[nodes[k]]; ++n; }
    if (n < 3) return 0;
    double ref = ln[0], dmax = -1e300, dmin = 1e300, lmax = -1e300, lmin = 1e300;
    for (int k = 0; k < n; ++k) {
        double d = wrap180(ln[k] - ref);
        if (d > dmax) dmax = d;
        if (d < dmin) dmin = d;
        if (la[k] > lmax) lmax = la[k];
        if (la[k] < lmin) lmin = la[k];
    }
    double dp = wrap180(lon_p - ref);
    if (dp > dmax || dp < dmin) return 0;
    if (lat_p > lmax || lat_p < lmin) return 0;
    double lo_min = ln[0], lo_max = ln[0];
    for (int k = 0; k < n; ++k) { if (ln[k] < lo_min) lo_min = ln[k]; if (ln[k] > lo_max) lo_max = ln[k]; }
    double lon0;
    if (lo_max - lo_min > 180.0) {
        double ds = 0.0;
        for (int k = 0; k < n; ++k) ds += wrap180(ln[k] - ln[0]);
        lon0 = ln[0] + ds / n;
    } else {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += ln[k];
        lon0 = s / n;
    }
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += la[k];
    double lat0 = s / n;
    double cl = cos(lat0 * DEG2RAD);
    double x[4], y[4];
    for (int k = 0; k < n; ++k) {
        x[k] = wrap180(ln[k] - lon0) * DEG2RAD * R_STD * cl;
        y[k] = (la[k] - lat0) * DEG2RAD * R_STD;
    }
    double px = wrap180(lon_p - lon0) * DEG2RAD * R_STD * cl;
    double py = (lat_p - lat0) * DEG2RAD * R_STD;
    double w[3];
    if (n == 3) {
        bary_tri(px, py, x, y, w);
        return w[0] >= BARY_EPS && w[1] >= BARY_EPS && w[2] >= BARY_EPS;
    }
    for (int i = 1; i < n - 1; ++i) {
        double tx[3] = {x[0], x[i], x[i + 1]}, ty[3] = {y[0], y[i], y[i + 1]};
        bary_tri(px, py, tx, ty, w);
        if (w[0] >= BARY_EPS && w[1] >= BARY_EPS && w[2] >= BARY_EPS) return 1;
    }
    return 0;
}

/* mesh.py:2392-2470 */
static int contain_local(const OMesh* m, double lon_p, double lat_p, int nn) {
    int cnt = m->n2e_cnt[nn];
    if (cnt == 0) return -1;
    const int32_t* row = m->n2e + (int64_t)nn * m->max_conn;
    for (int k = 0; k < cnt; ++k) {
        int c = row[k];
        if (c < 0) continue;
        if (element_contains(m, c, lon_p, lat_p)) return c;
    }
    for (int k = 0; k < cnt; ++k) {
        int e = row[k];
        if (e < 0) continue;
        for (int j = 0; j < m->max_v; ++j) {
            int v = m->en[(int64_t)e * m->max_v + j];
            if (v < 0 || v == nn) continue;
            int cv = m->n2e_cnt[v];
            const int32_t* rv = m->n2e + (int64_t)v * m->max_conn;
            for (int kk = 0; kk < cv; ++kk) {
                int c = rv[kk];
                if (c < 0) continue;
                int touches = 0;
                for (int jj = 0; jj < m->max_v; ++jj)
                    if (m->en[(int64_t)c * m->max_v + jj] == nn) { touches = 1; break; }
                if (touches) continue;
                if (element_contains(m, c, lon_p, lat_p)) return c;
            }
        }
    }
    return -1;
}

/* mesh.py:1973-2003 */
static double seam_lon0(const double* ln, int n) {
    double first = ln[0], lmin = first, lmax = first, s = 0.0;
    for (int v = 0; v < n; ++v) { s += ln[v]; if (ln[v] < lmin) lmin = ln[v]; if (ln[v] > lmax) lmax = ln[v]; }
    if (lmax - lmin > 180.0) {
        double d = 0.0;
        for (int v = 0; v < n; ++v) d += wrap180(ln[v] - first);
        return first + d / n;
    }
    return s / n;
}

/* interpolate.py:1404-1436, vertical.py:1042-1061 */
static double tblend(double a, double b, double t, double alpha0, double alpha) {
    if (alpha < 1e-12) {
        if (alpha0 == 0.0) return a;
        return (1.0 - alpha0) * a + alpha0 * b;
    }
    if (alpha > 1.0 - 1e-12) return t;
    if (alpha0 == 0.0) return (1.0 - alpha) * a + alpha * t;
    double a0 = (1.0 - alpha0) * a + alpha0 * b;
    return (1.0 - alpha) * a0 + alpha * t;
}

/* temporal_reconstruct.py:167-180 _fc_slope_scalar */
static double fc_slope(double dp, double dn, double hp, double hn) {
    if (dp * dn > 0.0) {
        double w1 = 2.0 * hn + hp, w2 = hn + 2.0 * hp;
        return (w1 + w2) / (w1 / dp + w2 / dn);
    }
    return 0.0;
}

/* temporal_reconstruct.py:183-215 _pchip_value_scalar: the monotone cubic
 * at tq in [t1, t2] */
static double pchip4(double f0, double f1, double f2, double f3, const double* t, double tq) {
    double h0 = t[1] - t[0], h1 = t[2] - t[1], h2 = t[3] - t[2];
    double d0 = (f1 - f0) / h0, d1 = (f2 - f1) / h1, d2 = (f3 - f2) / h2;
    double m1 = fc_slope(d0, d1, h0, h1), m2 = fc_slope(d1, d2, h1, h2);
    double s = (tq - t[1]) / h1, s2 = s * s, s3 = s2 * s;
    double h00 = 2.0 * s3 - 3.0 * s2 + 1.0, h10 = s3 - 2.0 * s2 + s, h01 = -2.0 * s3 + 3.0 * s2, h11 = s3 - s2;
    return h00 * f1 + h10 * h1 * m1 + h01 * f2 + h11 * h1 * m2;
}

/* the stage value of one field entry: the linear bracket blend, or the
 * PCHIP stencil at time `alpha` (make_stage_vels_recon) */
static double blend4(const OField* f, const void* a, const void* b, const void* t, const void* d, int64_t idx,
                     double alpha) {
    if (f->pchip) return pchip4(fld(a, f->f32, idx), fld(b, f->f32, idx), fld(t, f->f32, idx), fld(d, f->f32, idx),
                                f->pt, alpha);
    return tblend(fld(a, f->f32, idx), fld(b, f->f32, idx), fld(t, f->f32, idx), f->alpha0, alpha);
}

/* interpolate.py:1340-1529 (row 0: 2-D; row = layer: 3-D) */
/* The walk's pre-validated containing element for the next interpolation of
 * this thread (-1: search from the anchor), as interpolate.py:1246-1270
 * takes elem_hint. */
static _Thread_local int t_elem_hint = -1;

static int interp_lsq(const OMesh* m, const OField* f, double xp, double yp, int nn, double td, int row,
                      double alpha, double* U, double* V);
static int interp_edge_lsq(const OMesh* m, const OField* f, double xp, double yp, int nn, double td, int row,
                           double alpha, int bc, double* U, double* V);

static int interp_uv(const OMesh* m, const OField* f, double xp, double yp, int nn, double td, int row,
                     double alpha, double* U, double* V) {
    if (f->lsq >= 2) return interp_edge_lsq(m, f, xp, yp, nn, td, row, alpha, f->lsq - 2, U, V);
    if (f->lsq) return interp_lsq(m, f, xp, yp, nn, td, row, alpha, U, V);   /* element-layout u/v, row = layer */
    *U = 0.0; *V = 0.0;
    int elem = t_elem_hint >= 0 ? t_elem_hint : contain_local(m, xp, yp, nn);
    if (elem < 0) return 0;
    int verts[4], nv = 0;
    for (int k = 0; k < m->max_v; ++k) {
        int nd = m->en[(int64_t)elem * m->max_v + k];
        if (nd < 0) continue;
        if (nv > 0 && nd == verts[0]) continue;
        verts[nv++] = nd;
    }
    if (nv < 3) return 0;
    double R = m->r_earth;
    double lon_ref = m->lon[verts[0]], dsum = 0.0, lat0 = 0.0;
    for (int k = 0; k < nv; ++k) { dsum += wrap180(m->lon[verts[k]] - lon_ref); lat0 += m->lat[verts[k]]; }
    double lon0 = lon_ref + dsum / nv;
    lat0 /= nv;
    double cosl = cos(lat0 * DEG2RAD);
    double vx[4], vy[4];
    for (int k = 0; k < nv; ++k) {
        vx[k] = wrap180(m->lon[verts[k]] - lon0) * DEG2RAD * R * cosl;
        vy[k] = (m->lat[verts[k]] - lat0) * DEG2RAD * R;
    }
    double px = wrap180(xp - lon0) * DEG2RAD * R * cosl;
    double py = (yp - lat0) * DEG2RAD * R;
    double w[4];
    polygon_weights(px, py, vx, vy, nv, w);
    if (w[0] == -1.0) return 0;
    double Us = 0.0, Vs = 0.0;
    for (int k = 0; k < nv; ++k) {
        int64_t idx = (int64_t)row * f->n + verts[k];
        double un = blend4(f, f->ua, f->ub, f->ut, f->ud, idx, alpha);
        double vn = blend4(f, f->va, f->vb, f->vt, f->vd, idx, alpha);
        Us += w[k] * un;
        Vs += w[k] * vn;
    }
    *U = td * Us;
    *V = td * Vs;
    return 1;
}

/* vertical.py:39-91 */
static int find_layer(const OMesh* m, double z, double bottom) {
    int K = m->K;
    const double* zl = m->zlev;
    if (K < 2) return 0;
    if (z <= zl[0]) return 0;
    int max_layer = K - 2;
    for (int k = 0; k < K - 1; ++k)
        if (zl[k + 1] > bottom) { max_layer = k - 1 > 0 ? k - 1 : 0; break; }
    if (z >= bottom || z >= zl[max_layer + 1]) return max_layer;
    for (int k = 0; k <= max_layer; ++k)
        if (z < zl[k + 1]) return k;
    return max_layer;
}

static double wat(const OField* f, int k, int node, double alpha) {
    int64_t idx = (int64_t)k * f->n + node;
    return blend4(f, f->wa, f->wb, f->wt, f->wd, idx, alpha);
}

#define MAX_NEIGH 64   /* vertical.py:443 _MAX_NEIGHBOURS */

/* vertical.py:447-485 _collect_neighbour_nodes: the centre, then each
 * element's vertex slots in order, first occurrence only, at most 64. */
static int neigh_ring(const OMesh* m, int nn, int32_t* buf) {
    int count = 1;
    buf[0] = nn;
    int ne = m->n2e_cnt[nn];
    for (int k = 0; k < ne; ++k) {
        int e = m->n2e[(int64_t)nn * m->max_conn + k];
        if (e < 0) continue;
        for (int v = 0; v < m->max_v; ++v) {
            int nd = m->en[(int64_t)e * m->max_v + v];
            if (nd < 0) continue;
            int found = 0;
            for (int j = 0; j < count; ++j)
                if (buf[j] == nd) { found = 1; break; }
            if (!found && count < MAX_NEIGH) buf[count++] = nd;
        }
    }
    return count;
}

/* vertical.py:1064-1098 */
static double w_linear(const OMesh* m, const OField* f, double alpha, double z, int node, double td) {
    int K = m->K;
    const double* zl = m->zlev;
    if (K < 2) return td * wat(f, 0, node, alpha);
    if (z <= zl[0]) return td * wat(f, 0, node, alpha);
    if (z >= zl[K - 1]) return td * wat(f, K - 1, node, alpha);
    int k = K - 2;
    for (int j = 0; j < K - 1; ++j)
        if (z < zl[j + 1]) { k = j; break; }
    double dz = zl[k + 1] - zl[k];
    if (dz < 1e-12) return td * wat(f, k, node, alpha);
    double a = (z - zl[k]) / dz;
    double lo = wat(f, k, node, alpha), hi = wat(f, k + 1, node, alpha);
    return td * ((1.0 - a) * lo + a * hi);
}

static double pymin(double a, double b) { return b < a ? b : a; }

/* vertical.py:493-601 _interp_w_leastsq_single (w_code 2) and :1148-1229
 * _interp_w_idw_single (w_code 3) on the stage's W: the anchor's 1-ring of
 * nodes, each node's W at min(z, its bottom) */
static double w_ring(const OMesh* m, const OField* f, int w_code, double alpha, double xp, double yp, double z,
                     int node, double td) {
    int32_t buf[MAX_NEIGH];
    int count = neigh_ring(m, node, buf);
    double fallback = w_linear(m, f, alpha, pymin(z, m->depth[node]), node, td);
    double z0 = cos(yp * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    if (w_code == 3) {
        double sw = 0.0, swv = 0.0;
        for (int i = 0; i < count; ++i) {
            int nd = buf[i];
            double wv = w_linear(m, f, alpha, pymin(z, m->depth[nd]), nd, td);
            double dx = wrap180(m->lon[nd] - xp) * z0;
            double dy = (m->lat[nd] - yp) * SLM;
            double d2 = dx * dx + dy * dy;
            if (d2 < 1.0) return wv;
            double wt = 1.0 / d2;
            sw += wt;
            swv += wt * wv;
        }
        if (sw < 1e-30) return fallback;
        return swv / sw;
    }
    if (count < 3) return fallback;
    double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0, fw = 0.0, f1w = 0.0, f2w = 0.0;
    for (int i = 0; i < count; ++i) {
        int nd = buf[i];
        double wv = w_linear(m, f, alpha, pymin(z, m->depth[nd]), nd, td);
        double ex = wrap180(m->lon[nd] - xp) * z0;
        double ey = (m->lat[nd] - yp) * SLM;
        a11 += 1.0; a12 += ex; a13 += ey;
        a22 += ex * ex; a23 += ex * ey; a33 += ey * ey;
        fw += wv; f1w += wv * ex; f2w += wv * ey;
    }
    double a21 = a12, a31 = a13, a32 = a23;
    double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                 a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return fallback;
    double inv = 1.0 / fabs(det);
    double b11 = a22 * a33 - a23 * a32, b12 = a13 * a32 - a12 * a33, b13 = a12 * a23 - a13 * a22;
    return (b11 * fw + b12 * f1w + b13 * f2w) * inv;
}

/* vertical.py:744-881 */
static double w_bary(const OMesh* m, const OField* f, double alpha, double xp, double yp, double z, int node, double td) {
    int cnt = m->n2e_cnt[node];
    if (cnt == 0) return w_linear(m, f, alpha, pymin(z, m->depth[node]), node, td);
    for (int k = 0; k < cnt; ++k) {
        int e = m->n2e[(int64_t)node * m->max_conn + k];
        if (e < 0) continue;
        int verts[4], nv = 0;
        for (int v = 0; v < m->max_v; ++v) {
            int nd = m->en[(int64_t)e * m->max_v + v];
            if (nd < 0) continue;
            if (nv > 0 && nd == verts[0]) continue;
            verts[nv++] = nd;
        }
        if (nv < 3) continue;
        double ln[4];
        for (int v = 0; v < nv; ++v) ln[v] = m->lon[verts[v]];
        double lon0 = seam_lon0(ln, nv), lat0 = 0.0;
        for (int v = 0; v < nv; ++v) lat0 += m->lat[verts[v]];
        lat0 /= nv;
        double cl = cos(lat0 * DEG2RAD), R = 6371000.0;
        double vx[4], vy[4];
        for (int v = 0; v < nv; ++v) {
            vx[v] = wrap180(m->lon[verts[v]] - lon0) * DEG2RAD * R * cl;
            vy[v] = (m->lat[verts[v]] - lat0) * DEG2RAD * R;
        }
        double px = wrap180(xp - lon0) * DEG2RAD * R * cl;
        double py = (yp - lat0) * DEG2RAD * R;
        for (int t = 0; t < nv - 2; ++t) {
            int i1 = t + 1, i2 = t + 2;
            double ax = vx[0], ay = vy[0], bx = vx[i1], by = vy[i1], cx = vx[i2], cy = vy[i2];
            double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
            if (fabs(denom) < 1e-14) continue;
            double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
            double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
            double w3 = 1.0 - w1 - w2;
            if (w1 >= -1e-6 && w2 >= -1e-6 && w3 >= -1e-6) {
                if (nv == 4) {
                    double wts[4], acc = 0.0;
                    polygon_weights(px, py, vx, vy, 4, wts);
                    for (int vi = 0; vi < 4; ++vi)
                        acc += wts[vi] * w_linear(m, f, alpha, pymin(z, m->depth[verts[vi]]), verts[vi], td);
                    return acc;
                }
                int n0 = verts[0], n1 = verts[i1], n2 = verts[i2];
                double a0 = w_linear(m, f, alpha, pymin(z, m->depth[n0]), n0, td);
                double a1 = w_linear(m, f, alpha, pymin(z, m->depth[n1]), n1, td);
                double a2 = w_linear(m, f, alpha, pymin(z, m->depth[n2]), n2, td);
                return w1 * a0 + w2 * a1 + w3 * a2;
            }
        }
    }
    return w_linear(m, f, alpha, pymin(z, m->depth[node]), node, td);
}

/* W of one stage by the step's method (integrators.py:1260-1288 _compute_w, z-level) */
static double w_stage(const OMesh* m, const OField* f, int w_code, double alpha, double xp, double yp, double z,
                      int node, double td) {
    if (w_code == 0) return w_linear(m, f, alpha, z, node, td);
    if (w_code == 1) return w_bary(m, f, alpha, xp, yp, z, node, td);
    return w_ring(m, f, w_code, alpha, xp, yp, z, node, td);
}

/* diffusion.py:180-249 */
static uint64_t splitmix64(uint64_t x) {
    x = x + 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

uint64_t orc_key_hash(uint64_t k0, uint64_t k1, uint64_t k2, uint64_t k3, uint64_t k4) {
    uint64_t h = k0;
    h = splitmix64(h ^ k1);
    h = splitmix64(h ^ k2);
    h = splitmix64(h ^ k3);
    h = splitmix64(h ^ k4);
    return h;
}

void orc_normal_pair(uint64_t seed, uint64_t real_id, uint64_t pid, uint64_t step, uint64_t comp, double* g) {
    uint64_t h = orc_key_hash(seed, real_id, pid, step, comp);
    double inv = 1.0 / 4294967296.0, half = 0.5 * inv;
    double u1 = (double)((h >> 32) & 0xFFFFFFFFull) * inv + half;
    double u2 = (double)(h & 0xFFFFFFFFull) * inv + half;
    double two_pi = 2.0 * 3.141592653589793;
    double r = sqrt(-2.0 * log(u1));
    g[0] = r * cos(two_pi * u2);
    g[1] = r * sin(two_pi * u2);
}

/* diffusion.py:538-575 */
static void sphere_displace(double lon, double lat, double dx, double dy, double* lon2, double* lat2) {
    double dist = sqrt(dx * dx + dy * dy);
    if (dist == 0.0) { *lon2 = lon; *lat2 = lat; return; }
    double rm = SLM / DEG2RAD;
    double lam = lon * DEG2RAD, phi = lat * DEG2RAD;
    double cl = cos(lam), sl = sin(lam), cp = cos(phi), sp = sin(phi);
    double delta = dist / rm;
    double c = cos(delta), s = sin(delta) / dist;
    double tx = -sl * dx - sp * cl * dy;
    double ty = cl * dx - sp * sl * dy;
    double tz = cp * dy;
    double x2 = cp * cl * c + tx * s, y2 = cp * sl * c + ty * s, z2 = sp * c + tz * s;
    if (z2 > 1.0) z2 = 1.0;
    else if (z2 < -1.0) z2 = -1.0;
    *lat2 = asin(z2) / DEG2RAD;
    *lon2 = wrap180(atan2(y2, x2) / DEG2RAD);
}

typedef struct {
    int scheme, dims, w_code, kick;
    double dt, td, ak[4], kh_x, kh_y;
    uint64_t seed, real_id, step_i, pid_offset;
    int uv_dl;
    int az_on, az_field;   /* vertical Az kick; Az from the snapshots' (K, N) az arrays */
    double az_const;
    double Dmin, z0b_min;  /* sigma column floor and bed clearance */
    double alpha_end;      /* blend fraction of the end-of-step surface (sigma) */
    const double* eta_s;   /* sigma: the tracking layer's surface at the step's start (N), or NULL */
    const double* eta_e;   /* sigma: the tracking layer's surface at the step's end (N), or NULL */
    int sig_steady;        /* sigma: a steady step (stage surfaces blend from start to end) */
} OStep;

/* vertical_uv.py:457-523 uv_bracket */
static void uv_bracket(const double* p, int li, double z, int* k, double* alpha) {
    if (li <= 0) { *k = 0; *alpha = -1.0; return; }
    double zc = z;
    if (zc > p[li]) zc = p[li];
    if (zc < p[0]) zc = p[0];
    if (zc <= p[0]) { *k = 0; *alpha = -1.0; return; }
    if (zc >= p[li]) { *k = li; *alpha = -1.0; return; }
    int kk = li - 1;
    for (int j = 0; j < li; ++j)
        if (zc < p[j + 1]) { kk = j; break; }
    double dz = p[kk + 1] - p[kk];
    if (dz < 1e-12) { *k = kk; *alpha = -1.0; return; }
    double a = (zc - p[kk]) / dz;
    if (a <= 0.0) { *k = kk; *alpha = -1.0; return; }
    if (a >= 1.0) { *k = kk + 1; *alpha = -1.0; return; }
    *k = kk;
    *alpha = a;
}

/* interpolate.py:1847-1876 _tinterp_point_uv */
static void point_uv(const OField* f, int k, int nd, double alpha, double* u, double* v) {
    int64_t idx = (int64_t)k * f->n + nd;
    *u = blend4(f, f->ua, f->ub, f->ut, f->ud, idx, alpha);
    *v = blend4(f, f->va, f->vb, f->vt, f->vd, idx, alpha);
}

/* interpolate.py:1879-1971 _interp_barycentric_core_tinterp_dl with
 * :1664-1711 _dl_node_wall */
static int interp_uv_dl(const OMesh* m, const OField* f, double xp, double yp, int nn, double z, double td,
                        double alpha, double* U, double* V) {
    *U = 0.0; *V = 0.0;
    int elem = t_elem_hint >= 0 ? t_elem_hint : contain_local(m, xp, yp, nn);
    if (elem < 0) return 0;
    int verts[4], nv = 0;
    for (int k = 0; k < m->max_v; ++k) {
        int nd = m->en[(int64_t)elem * m->max_v + k];
        if (nd < 0) continue;
        if (nv > 0 && nd == verts[0]) continue;
        verts[nv++] = nd;
    }
    if (nv < 3) return 0;
    double R = m->r_earth;
    double lon_ref = m->lon[verts[0]], dsum = 0.0, lat0 = 0.0;
    for (int k = 0; k < nv; ++k) { dsum += wrap180(m->lon[verts[k]] - lon_ref); lat0 += m->lat[verts[k]]; }
    double lon0 = lon_ref + dsum / nv;
    lat0 /= nv;
    double cosl = cos(lat0 * DEG2RAD);
    double vx[4], vy[4];
    for (int k = 0; k < nv; ++k) {
        vx[k] = wrap180(m->lon[verts[k]] - lon0) * DEG2RAD * R * cosl;
        vy[k] = (m->lat[verts[k]] - lat0) * DEG2RAD * R;
    }
    double px = wrap180(xp - lon0) * DEG2RAD * R * cosl;
    double py = (yp - lat0) * DEG2RAD * R;
    double w[4];
    polygon_weights(px, py, vx, vy, nv, w);
    if (w[0] == -1.0) return 0;
    double zq = isnan(z) ? INFINITY : z;
    int wet[4], n_wet = 0;
    for (int k = 0; k < nv; ++k) { wet[k] = zq <= m->dl_bed[verts[k]]; n_wet += wet[k]; }
    if (n_wet == 0) {
        int kd = 0;
        for (int k = 1; k < nv; ++k)
            if (m->dl_bed[verts[k]] > m->dl_bed[verts[kd]]) kd = k;
        double un, vn;
        point_uv(f, m->dl_last[verts[kd]], verts[kd], alpha, &un, &vn);
        *U = td * un; *V = td * vn;
        return 1;
    }
    double den = 1.0;
    if (n_wet < nv) {
        double wsum = 0.0;
        for (int k = 0; k < nv; ++k)
            if (wet[k]) { if (w[k] < 0.0) w[k] = 0.0; wsum += w[k]; }
        if (wsum < 1e-12) {
            for (int k = 0; k < nv; ++k) if (wet[k]) w[k] = 1.0;
            den = (double)n_wet;
        } else den = wsum;
    }
    double Us = 0.0, Vs = 0.0;
    for (int k = 0; k < nv; ++k) {
        int nd = verts[k];
        if (n_wet < nv && !wet[k]) continue;
        int kb;
        double ab, un, vn;
        uv_bracket(m->dl_p, m->dl_last[nd], zq, &kb, &ab);
        point_uv(f, kb, nd, alpha, &un, &vn);
        if (!(ab < 0.0)) {
            double un1, vn1;
            point_uv(f, kb + 1, nd, alpha, &un1, &vn1);
            un = (1.0 - ab) * un + ab * un1;
            vn = (1.0 - ab) * vn + ab * vn1;
        }
        Us += w[k] * un; Vs += w[k] * vn;
    }
    if (n_wet < nv) { Us = Us / den; Vs = Vs / den; }
    *U = td * Us; *V = td * Vs;
    return 1;
}

/* u/v of a 3-D stage: the layer rule or the depth-linear rule */
static int stage_uv(const OMesh* m, const OField* f, const OStep* s, double xp, double yp, int nn, double z,
                    double alpha, double* U, double* V) {
    if (s->uv_dl) return interp_uv_dl(m, f, xp, yp, nn, z, s->td, alpha, U, V);
    return interp_uv(m, f, xp, yp, nn, s->td, find_layer(m, z, m->depth[nn]), alpha, U, V);
}

static double z0_of(double lat) {
    double z0 = cos(lat * DEG2RAD) * SLM;
    return z0 < 1.0 ? 1.0 : z0;
}
static double clat(double x) { return x > 90.0 ? 90.0 : (x < -90.0 ? -90.0 : x); }


/* diffusion.py:333-352 reflect_depth: specular fold into [top, bot] */
static double reflect_depth(double z, double top, double bot) {
    double L = bot - top;
    if (L <= 0.0) return top;
    double y = pymod(z - top, 2.0 * L);   /* 2L > 0: the positive-divisor fold */
    if (y < 0.0) y += 2.0 * L;
    if (y > L) y = 2.0 * L - y;
    return top + y;
}

/* the payload's Az at interface k of node (io.py:68-117 blend of the pair) */
static double az_at(const OField* f, int k, int node) {
    int64_t idx = (int64_t)k * f->n + node;
    double a = fld(f->aza, f->f32, idx);
    if (f->alpha0 == 0.0) return a;
    double b = fld(f->azb, f->f32, idx);
    return (1.0 - f->alpha0) * a + f->alpha0 * b;
}

/* diffusion.py:357-423 _az_interp_column + az_column_value_gradient */
static void az_column(const OMesh* m, const OField* f, int node, double z, double node_bottom, double* az,
                      double* g) {
    int K = m->K;
    const double* zl = m->zlev;
    double top = zl[0];
    double bot = node_bottom < zl[K - 1] ? node_bottom : zl[K - 1];
    if (bot < top) bot = top;
    double ze = z;
    if (ze < top) ze = top;
    if (ze > bot) ze = bot;
    double val;
    if (K < 2 || ze <= zl[0]) val = az_at(f, 0, node);
    else if (ze >= zl[K - 1]) val = az_at(f, K - 1, node);
    else {
        val = az_at(f, K - 1, node);
        for (int k = 0; k < K - 1; ++k)
            if (ze <= zl[k + 1]) {
                double dzl = zl[k + 1] - zl[k];
                if (dzl <= 0.0) { val = az_at(f, k, node); break; }
                double frac = (ze - zl[k]) / dzl;
                val = (1.0 - frac) * az_at(f, k, node) + frac * az_at(f, k + 1, node);
                break;
            }
    }
    *az = val;
    *g = 0.0;
    if (K < 2) return;
    int k = K - 2;
    for (int kk = 0; kk < K - 1; ++kk)
        if (ze <= zl[kk + 1]) { k = kk; break; }
    double dz = zl[k + 1] - zl[k];
    if (dz <= 0.0) return;
    if (f->f32 && f->alpha0 == 0.0) {
        /* an unblended float32 snapshot: the difference of two float32
           values rounds in float32 before the float64 division */
        float d = (float)az_at(f, k + 1, node) - (float)az_at(f, k, node);
        *g = (double)d / dz;
    } else {
        *g = (az_at(f, k + 1, node) - az_at(f, k, node)) / dz;
    }
}

/* integrators.py:842-938 _apply_split_az_kick with diffusion.py:302-330
 * diffusion_az_step_meters and :426-455 _loop_az_kick_zlevel, one particle */
static void az_kick(const OMesh* m, const OField* f, const OStep* s, int64_t pid, int nn, double* z) {
    double az, g;
    if (s->az_field) az_column(m, f, nn, *z, m->depth[nn], &az, &g);
    else { az = s->az_const; g = 0.0; }
    if (az < 0.0) { az = 0.0; g = 0.0; }
    double xi[2];
    orc_normal_pair(s->seed, s->real_id, (uint64_t)pid + s->pid_offset, s->step_i, 1, xi);
    double sdt = s->td * s->dt;
    double abs_dt = sdt >= 0.0 ? sdt : -sdt;
    double dz = g * abs_dt + sqrt(2.0 * az * abs_dt) * xi[0];
    *z = reflect_depth(*z + dz, m->zlev[0], m->depth[nn]);
}

/* integrators.py:917-930 with diffusion.py:458-482 _loop_az_kick_sigma, one
 * particle: the constant Az, no drift, folded into [0, max(H, Dmin) - z0b_min]
 * of its end-of-step column H */
static void az_kick_sigma(const OStep* s, int64_t pid, double H, double* z) {
    if (H < s->Dmin) H = s->Dmin;
    double bot = H - s->z0b_min;
    if (bot < 0.0) bot = 0.0;
    double xi[2];
    orc_normal_pair(s->seed, s->real_id, (uint64_t)pid + s->pid_offset, s->step_i, 1, xi);
    double sdt = s->td * s->dt;
    double abs_dt = sdt >= 0.0 ? sdt : -sdt;
    double dz = 0.0 * abs_dt + sqrt(2.0 * s->az_const * abs_dt) * xi[0];
    *z = reflect_depth(*z + dz, 0.0, bot);
}

/* integrators.py:673-818 for one surviving particle */
static void kick(const OMesh* m, const OStep* s, int64_t pid, double pre_lon, double pre_lat, double pre_z, int pre_nn,
                 double* lon, double* lat, double* z, int* status, int* nn, int8_t* fr, int is3d) {
    double g[2];
    orc_normal_pair(s->seed, s->real_id, (uint64_t)pid + s->pid_offset, s->step_i, 0, g);
    double adt = s->dt >= 0.0 ? s->dt : -s->dt;
    double sq = sqrt(adt), sx = sqrt(2.0 * s->kh_x), sy = sqrt(2.0 * s->kh_y);
    double dx = sx * sq * g[0], dy = sy * sq * g[1];
    if (s->kh_x != s->kh_y) {
        double la = *lat;
        if (la < -89.9) la = -89.9;
        if (la > 89.9) la = 89.9;
        dy = dy + (s->kh_x - s->kh_y) * tan(la * DEG2RAD) / (SLM / DEG2RAD) * adt;
    }
    double lk, lak;
    sphere_displace(*lon, *lat, dx, dy, &lk, &lak);
    int nk = anchor(m, lk, lak);
    if (contain_local(m, lk, lak, nk) < 0) {
        *status = OUTSIDE; *lon = pre_lon; *lat = pre_lat; *z = pre_z; *nn = pre_nn; *fr = 2;
        return;
    }
    *lon = lk; *lat = lak; *nn = nk;
    if (is3d) {
        double zv = *z;
        if (zv < m->zlev[0]) zv = m->zlev[0];
        if (zv > m->depth[nk]) zv = m->depth[nk];
        *z = zv;
    }
}

/* integrators.py:2521-2816 (2-D RK2/RK4 fused), the unfused Euler's per-particle
 * arithmetic (integrators.py:4997-5147), :3647-3856 (3-D RK2 fused). */
/* mesh.py:2488-2590 _walk_containing_element: from element e, cross the
 * edge of the most negative normalized signed-area coordinate until all are
 * >= -1e-6 (a near-edge accept below 1e-2 is verified with the exact local
 * predicate), at most 256 crossings; -1 for every non-contained outcome. */
static int edge_walk(const OMesh* m, double lon_p, double lat_p, int e) {
    if (e < 0 || e >= m->E || !m->enb) return -1;
    int prev = -1;
    for (int it = 0; it < 256; ++it) {
        int verts[4], nv = 0;
        for (int k = 0; k < m->max_v; ++k) {
            int nd = m->en[(int64_t)e * m->max_v + k];
            if (nd < 0) continue;
            if (nv > 0 && nd == verts[0]) continue;
            verts[nv++] = nd;
        }
        if (nv < 3) return -1;
        double ln[4], la[4];
        for (int k = 0; k < nv; ++k) { ln[k] = m->lon[verts[k]]; la[k] = m->lat[verts[k]]; }
        /* mesh.py:2006-2051 _project_to_local_xy */
        double lmin = ln[0], lmax = ln[0];
        for (int k = 0; k < nv; ++k) { if (ln[k] < lmin) lmin = ln[k]; if (ln[k] > lmax) lmax = ln[k]; }
        double lon0;
        if (lmax - lmin > 180.0) {
            double ds = 0.0;
            for (int k = 0; k < nv; ++k) ds += wrap180(ln[k] - ln[0]);
            lon0 = ln[0] + ds / nv;
        } else {
            double sm = 0.0;
            for (int k = 0; k < nv; ++k) sm += ln[k];
            lon0 = sm / nv;
        }
        double sl = 0.0;
        for (int k = 0; k < nv; ++k) sl += la[k];
        double lat0 = sl / nv;
        double cl = cos(lat0 * DEG2RAD);
        double x[4], y[4];
        for (int k = 0; k < nv; ++k) {
            x[k] = wrap180(ln[k] - lon0) * DEG2RAD * R_STD * cl;
            y[k] = (la[k] - lat0) * DEG2RAD * R_STD;
        }
        double px = wrap180(lon_p - lon0) * DEG2RAD * R_STD * cl;
        double py = (lat_p - lat0) * DEG2RAD * R_STD;
        double S = 0.0;
        for (int k = 0; k < nv; ++k) {
            int j = (k + 1) % nv;
            S += x[k] * y[j] - x[j] * y[k];
        }
        double absS = fabs(S);
        if (absS < AREA_TOL) return -1;
        double sgn = S > 0.0 ? 1.0 : -1.0;
        double worst = 1.0e100;
        int worst_k = -1;
        for (int k = 0; k < nv; ++k) {
            int j = (k + 1) % nv;
            double A = (x[j] - x[k]) * (py - y[k]) - (px - x[k]) * (y[j] - y[k]);
            double w = A * sgn / absS;
            if (w < worst) { worst = w; worst_k = k; }
        }
        if (worst >= -1e-6) {
            if (worst >= 1e-2) return e;
            return element_contains(m, e, lon_p, lat_p) ? e : -1;
        }
        int nb = m->enb[(int64_t)e * m->max_v + worst_k];
        if (nb < 0 || nb == prev) return -1;
        prev = e;
        e = nb;
    }
    return -1;
}

/* mesh.py:2593-2712 find_containing_elements_walk for one point: the walk
 * from the carried element, else the local scan around the widened anchor,
 * else around the exact anchor nn (the exactness heal); -1 outside. */
static int walk_locate(const OMesh* m, double lon_p, double lat_p, int start, int nn) {
    if (start >= 0) {
        int e = edge_walk(m, lon_p, lat_p, start);
        if (e >= 0) return e;
    }
    int nw = nearest_widened(m, lon_p, lat_p);
    int e = contain_local(m, lon_p, lat_p, nw);
    if (e >= 0) return e;
    return contain_local(m, lon_p, lat_p, nn);
}

/* ---- NEMO C-grid meshes (numerics/nemo_cgrid.py) ------------------- */

/* the stage's face value at flat raster index idx (the rasters of the
 * payload blended like every field, io.py:68-117) */
static double cg_val(const void* a, const void* b, const void* t, const OField* f, int64_t idx, double alpha) {
    return tblend(fld(a, f->f32, idx), fld(b, f->f32, idx), fld(t, f->f32, idx), f->alpha0, alpha);
}

/* nemo_cgrid.py:75-81 _nemo_cgrid_e3face */
static double cg_e3face(const OMesh* m, const int32_t* kb, const double* e3, int64_t fi, int k) {
    if (k == kb[fi]) return e3[fi];
    return m->cg_zw[k + 1] - m->cg_zw[k];
}

static double pmax(double a, double b) { return b > a ? b : a; }   /* Python max(a, b) */
static double pmin2(double a, double b) { return b < a ? b : a; }  /* Python min(a, b) */

/* nemo_cgrid.py:84-222 _interp_nemo_cgrid_core: the cell (hint >= 0, else
 * the local search around nn), the closed-form bilinear inverse, the face
 * fluxes (model widths, or each edge's plane length), the logical velocity
 * linear along its own axis; 3-D: zp is the fractional level s, W = ds/dt. */
static int cgrid_core(const OMesh* m, const OField* f, double alpha, double xp, double yp, double zp, int nn, int hint,
                      double td, int three_d, double* U, double* V, double* W) {
    *U = 0.0; *V = 0.0; *W = 0.0;
    int e = hint;
    if (e < 0) {
        e = contain_local(m, xp, yp, nn);
        if (e < 0) return 0;
    }
    if (m->cg_nlev[e] <= 0) return 1;
    const int64_t nx = m->cg_nx;
    const int64_t c = m->cg_ji[2 * (int64_t)e] * nx + m->cg_ji[2 * (int64_t)e + 1];
    int kz = 0;
    int64_t nynx = 0;
    double fW = 1.0, fE = 1.0, fS = 1.0, fN = 1.0, e3c = 1.0;
    if (three_d) {
        nynx = m->cg_nynx;
        if (zp >= m->cg_nlev[e]) return 1;
        kz = (int)floor(zp);
        if (kz < 0) kz = 0;
        if (kz > m->cg_K - 1) kz = m->cg_K - 1;
        e3c = m->cg_zw[kz + 1] - m->cg_zw[kz];
        if (kz == m->cg_nlev[e] - 1) e3c = m->cg_e3b[c];
        fW = cg_e3face(m, m->cg_kbu, m->cg_e3u, c - 1, kz) / e3c;
        fE = cg_e3face(m, m->cg_kbu, m->cg_e3u, c, kz) / e3c;
        fS = cg_e3face(m, m->cg_kbv, m->cg_e3v, c - nx, kz) / e3c;
        fN = cg_e3face(m, m->cg_kbv, m->cg_e3v, c, kz) / e3c;
    }
    const int64_t ko = (int64_t)kz * nynx;
    double uW = cg_val(f->ua, f->ub, f->ut, f, ko + c - 1, alpha);
    double uE = cg_val(f->ua, f->ub, f->ut, f, ko + c, alpha);
    double vS = cg_val(f->va, f->vb, f->vt, f, ko + c - nx, alpha);
    double vN = cg_val(f->va, f->vb, f->vt, f, ko + c, alpha);
    const double M = SLM;
    double cosl = cos(yp * DEG2RAD);
    double px[4], py[4];
    for (int k = 0; k < 4; ++k) {
        int nd = m->cg_corners[4 * (int64_t)e + k];
        px[k] = wrap180(m->lon[nd] - xp) * cosl * M;
        py[k] = (m->lat[nd] - yp) * M;
    }
    double a0 = px[0], a1 = px[1] - px[0], a2 = px[3] - px[0], a3 = px[0] - px[1] + px[2] - px[3];
    double b0 = py[0], b1 = py[1] - py[0], b2 = py[3] - py[0], b3 = py[0] - py[1] + py[2] - py[3];
    double scale = pmax(pmax(pmax(pmax(fabs(a1), fabs(a2)), fabs(b1)), fabs(b2)), 1e-30);
    double aa = a3 * b2 - a2 * b3;
    double bb = a3 * b0 - a0 * b3 + a1 * b2 - a2 * b1;
    double cc = a1 * b0 - a0 * b1;
    double eta;
    if (fabs(aa) < 1e-12 * scale * scale) {
        if (fabs(bb) < 1e-300) return 0;
        eta = -cc / bb;
    } else {
        double disc = bb * bb - 4.0 * aa * cc;
        if (disc < 0.0) disc = 0.0;
        double sq = sqrt(disc);
        double r1 = (-bb + sq) / (2.0 * aa);
        double r2 = (-bb - sq) / (2.0 * aa);
        double d1 = pmax(pmax(0.0, -r1), r1 - 1.0);
        double d2 = pmax(pmax(0.0, -r2), r2 - 1.0);
        eta = d1 <= d2 ? r1 : r2;
    }
    eta = pmin2(pmax(eta, 0.0), 1.0);
    double den = a1 + a3 * eta, den2 = b1 + b3 * eta;
    double xi;
    if (fabs(den) >= fabs(den2)) xi = (0.0 - a0 - a2 * eta) / den;
    else xi = (0.0 - b0 - b2 * eta) / den2;
    xi = pmin2(pmax(xi, 0.0), 1.0);
    double U0, U1, V0, V1;
    if (m->cg_has_e) {
        U0 = fW * uW * m->cg_e2u[c - 1]; U1 = fE * uE * m->cg_e2u[c];
        V0 = fS * vS * m->cg_e1v[c - nx]; V1 = fN * vN * m->cg_e1v[c];
    } else {
        double L[4];
        for (int k = 0; k < 4; ++k) {
            int na = m->cg_corners[4 * (int64_t)e + k], nb = m->cg_corners[4 * (int64_t)e + (k + 1) % 4];
            double dl = wrap180(m->lon[nb] - m->lon[na]);
            double cm = cos(0.5 * (m->lat[na] + m->lat[nb]) * DEG2RAD);
            L[k] = hypot(dl * cm * M, (m->lat[nb] - m->lat[na]) * M);
        }
        U0 = fW * uW * L[3]; U1 = fE * uE * L[1]; V0 = fS * vS * L[0]; V1 = fN * vN * L[2];
    }
    double dxdxi = (1.0 - eta) * a1 + eta * (px[2] - px[3]);
    double dydxi = (1.0 - eta) * b1 + eta * (py[2] - py[3]);
    double dxdeta = (1.0 - xi) * a2 + xi * (px[2] - px[1]);
    double dydeta = (1.0 - xi) * b2 + xi * (py[2] - py[1]);
    double det = dxdxi * dydeta - dxdeta * dydxi;
    double adet = fabs(det);
    if (adet < 1e-12 * scale * scale) return 0;
    double dxi = ((1.0 - xi) * U0 + xi * U1) / adet;
    double deta = ((1.0 - eta) * V0 + eta * V1) / adet;
    double Uv = dxdxi * dxi + dxdeta * deta;
    double Vv = dydxi * dxi + dydeta * deta;
    double Wv = 0.0;
    if (three_d) {
        double zeta = pmin2(pmax(zp - kz, 0.0), 1.0);
        Wv = ((1.0 - zeta) * cg_val(f->wa, f->wb, f->wt, f, ko + c, alpha)
              + zeta * cg_val(f->wa, f->wb, f->wt, f, ko + nynx + c, alpha)) * m->cg_area[c] / (adet * e3c);
    }
    *U = td * Uv; *V = td * Vv; *W = td * Wv;
    return 1;
}

/* nemo_cgrid.py:391-402 _cell_thickness */
static void cg_cell(const OMesh* m, int e, int ok, int k, int* kout, double* e3) {
    int64_t c = ok ? m->cg_ji[2 * (int64_t)e] * m->cg_nx + m->cg_ji[2 * (int64_t)e + 1] : 0;
    int nl = m->cg_nlev_r[c];
    if (k < 0) k = 0;
    if (k > m->cg_K - 1) k = m->cg_K - 1;
    *kout = k;
    *e3 = (k == nl - 1 && m->cg_shrunk) ? m->cg_e3b[c] : m->cg_zw[k + 1] - m->cg_zw[k];
}

/* nemo_cgrid.py:405-413 _level_coord, z -> s and s -> z */
static double cg_z2s(const OMesh* m, int e, int ok, double z) {
    int k = 0;
    if (isnan(z)) k = m->cg_K;
    else while (k < m->cg_K + 1 && m->cg_zw[k] <= z) ++k;
    double e3;
    cg_cell(m, e, ok, k - 1, &k, &e3);
    return k + (z - m->cg_zw[k]) / e3;
}
static double cg_s2z(const OMesh* m, int e, int ok, double s) {
    int k;
    double e3;
    cg_cell(m, e, ok, (int)floor(s), &k, &e3);
    return m->cg_zw[k] + (s - k) * e3;
}

/* nemo_cgrid.py:416-512 nemo_cgrid3d_step for one particle: Euler / RK2
 * (midpoint) / RK4 in the fractional level s = k + zeta of the start cell,
 * stage n at x0 + a_n k_{n-1}, the weighted sum of the stage increments,
 * s clamped at the surface, the end cell's domain check and s -> z; a
 * particle that is not alive only gets the nearest node of its position. */
static void step_cgrid3d(const OMesh* m, const OField* f, const OStep* s, int64_t i, double* lon, double* lat,
                         double* z, int* status, int* nn, int8_t* fr, double* U, double* V, double* W) {
    static const double A[3][4] = {{0.0}, {0.0, 0.5}, {0.0, 0.5, 0.5, 1.0}};
    static const double B[3][4] = {{1.0}, {0.0, 1.0}, {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6}};
    const int ns = s->scheme == 0 ? 1 : (s->scheme == 1 ? 2 : 4);
    double lon0 = lon[i], lat0 = lat[i], z0 = z[i], dt = s->dt;
    int nn0 = anchor(m, lon0, lat0);
    if (status[i] != ALIVE) {
        U[i] = 0.0; V[i] = 0.0; W[i] = 0.0;
        nn[i] = nn0;
        return;
    }
    int e0 = contain_local(m, lon0, lat0, nn0);
    int ok0 = e0 >= 0;
    double s0 = cg_z2s(m, e0, ok0, z0);
    double ks[4][3], first[3] = {0.0, 0.0, 0.0};
    int ok = 1;
    for (int n = 0; n < ns; ++n) {
        double ln = lon0, lt = lat0, sn = s0;
        if (n) {
            ln = wrap180(lon0 + A[s->scheme][n] * ks[n - 1][0]);
            lt = clat(lat0 + A[s->scheme][n] * ks[n - 1][1]);
            sn = s0 + A[s->scheme][n] * ks[n - 1][2];
        }
        double Un = 0.0, Vn = 0.0, Wn = 0.0;
        if (ok) {
            int nnn = n ? anchor(m, ln, lt) : nn0;
            int okn = cgrid_core(m, f, s->ak[n], ln, lt, sn, nnn, n ? -1 : (ok0 ? e0 : -1), s->td, 1, &Un, &Vn, &Wn);
            ok = ok && okn;
        }
        if (n == 0) { first[0] = Un; first[1] = Vn; first[2] = Wn; }
        ks[n][0] = dt * Un / z0_of(lt);
        ks[n][1] = dt * Vn / SLM;
        ks[n][2] = dt * Wn;
    }
    double d[3];
    for (int c = 0; c < 3; ++c) {
        d[c] = 0.0;
        for (int n = 0; n < ns; ++n) d[c] += B[s->scheme][n] * ks[n][c];
    }
    double ln = lon0, lt = lat0, sv = s0;
    if (ok) {
        ln = wrap180(lon0 + d[0]);
        lt = clat(lat0 + d[1]);
        sv = s0 + d[2];
        if (!(sv >= 0.0)) sv = isnan(sv) ? sv : 0.0;
    }
    int nne = anchor(m, ln, lt);
    int e1 = contain_local(m, ln, lt, nne);
    int in_dom = e1 >= 0;
    int failed = !ok || !in_dom;
    double zn = z0;
    int st = ALIVE;
    int8_t frr = fr[i];
    if (failed) {
        ln = lon0; lt = lat0; sv = s0; nne = nn0; st = OUTSIDE;
        frr = !ok ? 1 : 2;
    } else if (!(sv == s0 && e1 == e0)) {
        zn = cg_s2z(m, e1, in_dom, sv);
    }
    int kk;
    double e3;
    cg_cell(m, e0, ok0, (int)floor(s0), &kk, &e3);
    U[i] = first[0]; V[i] = first[1]; W[i] = first[2] * e3;
    lon[i] = ln; lat[i] = lt; z[i] = zn;
    status[i] = st; nn[i] = nne; fr[i] = frr;
}

/* interpolate.py:207-354 _interp_leastsq_core_tinterp (steady: :52-205;
 * PCHIP: :355-474): the plane a0 + a1 x + a2 y fitted through the anchor's
 * element-centre velocities (metres, centred on the particle, the seam gate
 * on the raw longitude difference), Cramer's rule, its value a0 at the
 * particle; 0 for an empty ring or a singular normal matrix. */
static int interp_lsq(const OMesh* m, const OField* f, double xp, double yp, int nn, double td, int row,
                      double alpha, double* U, double* V) {
    *U = 0.0; *V = 0.0;
    int count = m->n2e_cnt[nn];
    if (count < 1) return 0;
    double z0 = cos(yp * DEG2RAD) * SLM;
    double xp_m = xp * z0, yp_m = yp * SLM;
    double s11 = 0, s12 = 0, s13 = 0, s22 = 0, s23 = 0, s33 = 0, fu = 0, fu1 = 0, fu2 = 0, fv = 0, fv1 = 0, fv2 = 0;
    for (int k = 0; k < count; ++k) {
        int e = m->n2e[(int64_t)nn * m->max_conn + k];
        double ex = m->ec_lon[e] * z0 - xp_m;
        double raw = m->ec_lon[e] - xp;
        if (raw > 180.0) ex -= 360.0 * z0;
        else if (raw < -180.0) ex += 360.0 * z0;
        double ey = m->ec_lat[e] * SLM - yp_m;
        int64_t idx = (int64_t)row * f->n + e;
        double uu = td * blend4(f, f->ua, f->ub, f->ut, f->ud, idx, alpha);
        double vv = td * blend4(f, f->va, f->vb, f->vt, f->vd, idx, alpha);
        s11 = s11 + 1.0; s12 = s12 + ex; s13 = s13 + ey;
        s22 = s22 + ex * ex; s23 = s23 + ex * ey; s33 = s33 + ey * ey;
        fu = fu + uu; fu1 = fu1 + uu * ex; fu2 = fu2 + uu * ey;
        fv = fv + vv; fv1 = fv1 + vv * ex; fv2 = fv2 + vv * ey;
    }
    double s21 = s12, s31 = s13, s32 = s23;
    double det = s11 * s22 * s33 + s12 * s23 * s31 + s13 * s21 * s32 - s13 * s22 * s31 - s12 * s21 * s33 -
                 s11 * s23 * s32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(s11 * s22 * s33)) return 0;
    double inv = 1.0 / fabs(det);
    double c11 = s22 * s33 - s23 * s32, c12 = s13 * s32 - s12 * s33, c13 = s12 * s23 - s13 * s22;
    *U = (c11 * fu + c12 * fu1 + c13 * fu2) * inv;
    *V = (c11 * fv + c12 * fv1 + c13 * fv2) * inv;
    return 1;
}

/* interpolate.py:2588-2747 _interp_edge_leastsq_core (bc 0 freeslip, 1
 * noslip): the containing element, its centre and its edge neighbours'
 * centres (boundary edges: the mirrored centre and ghost velocity) */
static int interp_edge_lsq(const OMesh* m, const OField* f, double xp, double yp, int nn, double td, int row,
                           double alpha, int bc, double* U, double* V) {
    *U = 0.0; *V = 0.0;
    int el = contain_local(m, xp, yp, nn);
    if (el < 0) return 0;
    int verts[4], nv = 0;
    for (int k = 0; k < m->max_v; ++k) {
        int nd = m->en[(int64_t)el * m->max_v + k];
        if (nd < 0) continue;
        if (nv > 0 && nd == verts[0]) continue;
        verts[nv++] = nd;
    }
    if (nv < 3) return 0;
    double z0 = cos(yp * DEG2RAD) * SLM;
    double cx = wrap180(m->ec_lon[el] - xp) * z0, cy = (m->ec_lat[el] - yp) * SLM;
    int64_t io = (int64_t)row * f->n + el;
    double u_own = td * blend4(f, f->ua, f->ub, f->ut, f->ud, io, alpha);
    double v_own = td * blend4(f, f->va, f->vb, f->vt, f->vd, io, alpha);
    double a11 = 1.0, a12 = cx, a13 = cy, a22 = cx * cx, a23 = cx * cy, a33 = cy * cy;
    double fu = u_own, fu1 = u_own * cx, fu2 = u_own * cy, fv = v_own, fv1 = v_own * cx, fv2 = v_own * cy;
    for (int k = 0; k < nv; ++k) {
        int nb = m->enb[(int64_t)el * m->max_v + k];
        double ex, ey, uu, vv;
        if (nb >= 0) {
            ex = wrap180(m->ec_lon[nb] - xp) * z0;
            ey = (m->ec_lat[nb] - yp) * SLM;
            int64_t ib = (int64_t)row * f->n + nb;
            uu = td * blend4(f, f->ua, f->ub, f->ut, f->ud, ib, alpha);
            vv = td * blend4(f, f->va, f->vb, f->vt, f->vd, ib, alpha);
        } else {
            int na = verts[k], n2 = verts[(k + 1) % nv];
            double dax = wrap180(m->lon[na] - xp) * z0, day = (m->lat[na] - yp) * SLM;
            double dbx = wrap180(m->lon[n2] - xp) * z0, dby = (m->lat[n2] - yp) * SLM;
            double tx = dbx - dax, ty = dby - day, tt = tx * tx + ty * ty;
            if (tt <= 0.0) continue;
            double proj = ((cx - dax) * tx + (cy - day) * ty) / tt;
            double fx = dax + proj * tx, fy = day + proj * ty;
            ex = 2.0 * fx - cx;
            ey = 2.0 * fy - cy;
            if (bc == 1) { uu = -u_own; vv = -v_own; }
            else {
                double ut = (u_own * tx + v_own * ty) / tt;
                uu = 2.0 * ut * tx - u_own;
                vv = 2.0 * ut * ty - v_own;
            }
        }
        a11 = a11 + 1.0; a12 = a12 + ex; a13 = a13 + ey;
        a22 = a22 + ex * ex; a23 = a23 + ex * ey; a33 = a33 + ey * ey;
        fu = fu + uu; fu1 = fu1 + uu * ex; fu2 = fu2 + uu * ey;
        fv = fv + vv; fv1 = fv1 + vv * ex; fv2 = fv2 + vv * ey;
    }
    double a21 = a12, a31 = a13, a32 = a23;
    double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                 a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return 0;
    double inv = 1.0 / fabs(det);
    double c11 = a22 * a33 - a23 * a32, c12 = a13 * a32 - a12 * a33, c13 = a12 * a23 - a13 * a22;
    *U = (c11 * fu + c12 * fu1 + c13 * fu2) * inv;
    *V = (c11 * fv + c12 * fv1 + c13 * fv2) * inv;
    return 1;
}

/* u/v of a 2-D stage: the C-grid core on the surface faces
 * (nemo_cgrid.py:355-388 interp_nemo_cgrid), the element-centre least
 * squares, else the barycentric core */
static int uv2(const OMesh* m, const OField* f, double xp, double yp, int nn, double td, double alpha, double* U,
               double* V) {
    if (f->lsq >= 2) return interp_edge_lsq(m, f, xp, yp, nn, td, 0, alpha, f->lsq - 2, U, V);
    if (f->lsq) return interp_lsq(m, f, xp, yp, nn, td, 0, alpha, U, V);
    if (m->cg) {
        double Wd;
        int h = t_elem_hint;
        return cgrid_core(m, f, alpha, xp, yp, 0.0, nn, h, td, 0, U, V, &Wd);
    }
    return interp_uv(m, f, xp, yp, nn, td, 0, alpha, U, V);
}

/* Walk mode (elem_search: walk, elem != NULL): each stage's containing
 * element is walked from the previous stage's (the step's start from the
 * carried one) and handed to the interpolation as its element hint; the
 * end-of-step walk gives the domain verdict and the new carried element;
 * a failed step keeps the start element (integrators.py:5019-5147,
 * :5415-5608, :5792-6011). */
#define STAGE(e, call) (t_elem_hint = (e), _r = (call), t_elem_hint = -1, _r)

/* ---- sigma meshes (vertical_coord "sigma"; vertical_sigma.py,
 * integrators.py:1322-1440): the step integrates s = z / H_p, H_p the
 * column height max(depth + eta, Dmin) interpolated at the particle like W. */

/* the stage's free surface at a node: the payload's eta blended like u/v
 * (io.py:68-117 _blend in float64, the stage lerps of _make_stage_vels) */
static double eta_at(const OField* f, int node, double alpha) {
    if (f->pchip) return pchip4(f->etaa[node], f->etab[node], f->etat[node], f->etad[node], f->pt, alpha);
    return tblend(f->etaa[node], f->etab[node], f->etat[node], f->alpha0, alpha);
}

/* The surface at one instant of the step (integrators.py:1358-1441 and the
 * sigma branches :5031-5079, :5424-5436, :5797-5815): slot 0 the start, 1..3
 * the RK stages (c = 0.5, 0.5, 1), 4 the end; the tracking layer's surfaces
 * (eta_s, eta_e) where given, a steady step's stages blended from the start
 * to the end surface by _eta_blend, else the stage field's own. */
static double stage_alpha(const OStep* s, int slot) { return slot == 4 ? s->alpha_end : s->ak[slot]; }

static double eta_slot(const OField* f, const OStep* s, int node, int slot) {
    double e0 = s->eta_s ? s->eta_s[node] : eta_at(f, node, s->ak[0]);
    if (slot == 0) return e0;
    if (slot == 4 && s->eta_e) return s->eta_e[node];
    if (!s->sig_steady) return eta_at(f, node, stage_alpha(s, slot));
    double e1 = s->eta_e ? s->eta_e[node] : e0;
    if (slot == 3 || slot == 4) return e1;
    return (1.0 - 0.5) * e0 + 0.5 * e1;
}

/* vertical_sigma.py:472-478 _col_H */
static double col_H(const OMesh* m, const OField* f, const OStep* s, int node, int slot) {
    double H = m->depth[node] + eta_slot(f, s, node, slot);
    if (H < s->Dmin) H = s->Dmin;
    return H;
}

/* vertical_sigma.py:565-632 _bary_locate: the W search's element among the
 * anchor's elements and its vertex weights (tris: the fan triangle's, quads:
 * Wachspress); returns the vertex count, 0 when none contains the point. */
static int bary_locate(const OMesh* m, double xp, double yp, int node, int* verts, double* wts) {
    int cnt = m->n2e_cnt[node];
    for (int k = 0; k < cnt; ++k) {
        int e = m->n2e[(int64_t)node * m->max_conn + k];
        if (e < 0) continue;
        int nv = 0;
        for (int v = 0; v < m->max_v; ++v) {
            int nd = m->en[(int64_t)e * m->max_v + v];
            if (nd < 0) continue;
            if (nv > 0 && nd == verts[0]) continue;
            verts[nv++] = nd;
        }
        if (nv < 3) continue;
        double ln[4];
        for (int v = 0; v < nv; ++v) ln[v] = m->lon[verts[v]];
        double lon0 = seam_lon0(ln, nv), lat0 = 0.0;
        for (int v = 0; v < nv; ++v) lat0 += m->lat[verts[v]];
        lat0 /= nv;
        double cl = cos(lat0 * DEG2RAD), R = 6371000.0;
        double vx[4], vy[4];
        for (int v = 0; v < nv; ++v) {
            vx[v] = wrap180(m->lon[verts[v]] - lon0) * DEG2RAD * R * cl;
            vy[v] = (m->lat[verts[v]] - lat0) * DEG2RAD * R;
        }
        double px = wrap180(xp - lon0) * DEG2RAD * R * cl;
        double py = (yp - lat0) * DEG2RAD * R;
        for (int t = 0; t < nv - 2; ++t) {
            double ax = vx[0], ay = vy[0], bx = vx[t + 1], by = vy[t + 1], cx = vx[t + 2], cy = vy[t + 2];
            double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
            if (fabs(denom) < 1e-14) continue;
            double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
            double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
            double w3 = 1.0 - w1 - w2;
            if (w1 >= -1e-6 && w2 >= -1e-6 && w3 >= -1e-6) {
                for (int v = 0; v < 4; ++v) wts[v] = 0.0;
                if (nv == 4) polygon_weights(px, py, vx, vy, 4, wts);
                else { wts[0] = w1; wts[t + 1] = w2; wts[t + 2] = w3; }
                return nv;
            }
        }
    }
    return 0;
}

/* vertical_sigma.py:1034-1060 the particle's column height, interpolated
 * with the W method (nearest: the anchor's column; barycentric: :636-652) */
/* vertical_sigma.py:493-563 _H_leastsq_single (w_code 2) / _H_idw_single (3) */
static double H_ring(const OMesh* m, const OField* f, const OStep* s, int slot, double xp, double yp, int node) {
    int32_t buf[MAX_NEIGH];
    int count = neigh_ring(m, node, buf);
    double z0 = cos(yp * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    if (s->w_code == 3) {
        double sw = 0.0, swh = 0.0;
        for (int i = 0; i < count; ++i) {
            int nd = buf[i];
            double h = col_H(m, f, s, nd, slot);
            double dx = wrap180(m->lon[nd] - xp) * z0, dy = (m->lat[nd] - yp) * SLM;
            double d2 = dx * dx + dy * dy;
            if (d2 < 1.0) return h;
            sw += 1.0 / d2;
            swh += h / d2;
        }
        if (sw < 1e-30) return col_H(m, f, s, node, slot);
        return swh / sw;
    }
    if (count < 3) return col_H(m, f, s, node, slot);
    double a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, fw = 0, f1w = 0, f2w = 0;
    for (int i = 0; i < count; ++i) {
        int nd = buf[i];
        double h = col_H(m, f, s, nd, slot);
        double ex = wrap180(m->lon[nd] - xp) * z0, ey = (m->lat[nd] - yp) * SLM;
        a11 += 1.0; a12 += ex; a13 += ey; a22 += ex * ex; a23 += ex * ey; a33 += ey * ey;
        fw += h; f1w += h * ex; f2w += h * ey;
    }
    double a21 = a12, a31 = a13, a32 = a23;
    double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                 a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return col_H(m, f, s, node, slot);
    double inv = 1.0 / fabs(det);
    double H = ((a22 * a33 - a23 * a32) * fw + (a13 * a32 - a12 * a33) * f1w + (a12 * a23 - a13 * a22) * f2w) * inv;
    if (H < s->Dmin) H = s->Dmin;
    return H;
}

static double sigma_H(const OMesh* m, const OField* f, const OStep* s, int slot, double xp, double yp, int node) {
    if (s->w_code >= 2) return H_ring(m, f, s, slot, xp, yp, node);
    if (s->w_code == 0) return col_H(m, f, s, node, slot);
    int verts[4];
    double wts[4];
    int nv = bary_locate(m, xp, yp, node, verts, wts);
    if (nv == 0) return col_H(m, f, s, node, slot);
    double H = 0.0;
    for (int v = 0; v < nv; ++v) H += wts[v] * col_H(m, f, s, verts[v], slot);
    return H;
}

/* vertical_sigma.py:297-334 _interp_w_sigma_linear_single on the stage's w */
static double w_sig_linear(const OMesh* m, const OField* f, double alpha, double z, int node, double H, double td) {
    int K = m->K;
    const double* sg = m->sigma;
    if (K < 2) return td * wat(f, 0, node, alpha);
    double z_top = (1.0 - sg[0]) * H, z_bot = (1.0 - sg[K - 1]) * H;
    if (z <= z_top) return td * wat(f, 0, node, alpha);
    if (z >= z_bot) return td * wat(f, K - 1, node, alpha);
    int k = K - 2;
    for (int j = 0; j < K - 1; ++j)
        if (z < (1.0 - sg[j + 1]) * H) { k = j; break; }
    double zk = (1.0 - sg[k]) * H, zk1 = (1.0 - sg[k + 1]) * H;
    double dz = zk1 - zk;
    if (dz < 1e-12) return td * wat(f, k, node, alpha);
    double a = (z - zk) / dz;
    double wv = (1.0 - a) * wat(f, k, node, alpha) + a * wat(f, k + 1, node, alpha);
    return td * wv;
}

/* vertical_sigma.py:481-489 _sigma_frac */
static double sigma_frac(double z, double H) {
    double fr = z / H;
    if (fr < 0.0) fr = 0.0;
    else if (fr > 1.0) fr = 1.0;
    return fr;
}

/* W on a sigma mesh (vertical_sigma.py:971-1031): nearest = the anchor's
 * column (:337-360); barycentric = every vertex column at the particle's
 * sigma (:766-816), the own column at min(z, H) outside every element */
/* vertical_sigma.py:656-765 _interp_w_sigma_leastsq_single / :820-905
 * _interp_w_sigma_idw_single: the 1-ring sampled at the particle's sigma */
static double w_sig_ring(const OMesh* m, const OField* f, const OStep* s, int slot, double alpha, double xp, double yp,
                         double z, int node) {
    int32_t buf[MAX_NEIGH];
    int count = neigh_ring(m, node, buf);
    double Hn = col_H(m, f, s, node, slot);
    double fallback = w_sig_linear(m, f, alpha, z < Hn ? z : Hn, node, Hn, s->td);
    if (s->w_code == 2 && count < 3) return fallback;
    double z0 = cos(yp * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    double fr = sigma_frac(z, H_ring(m, f, s, slot, xp, yp, node));
    double a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, fw = 0, f1w = 0, f2w = 0, sw = 0, swv = 0;
    for (int i = 0; i < count; ++i) {
        int nd = buf[i];
        double H = col_H(m, f, s, nd, slot);
        double wv = w_sig_linear(m, f, alpha, fr * H, nd, H, s->td);
        double dx = wrap180(m->lon[nd] - xp) * z0, dy = (m->lat[nd] - yp) * SLM;
        if (s->w_code == 3) {
            double d2 = dx * dx + dy * dy;
            if (d2 < 1.0) return wv;
            double wt = 1.0 / d2;
            sw += wt;
            swv += wt * wv;
            continue;
        }
        a11 += 1.0; a12 += dx; a13 += dy; a22 += dx * dx; a23 += dx * dy; a33 += dy * dy;
        fw += wv; f1w += wv * dx; f2w += wv * dy;
    }
    if (s->w_code == 3) return sw < 1e-30 ? fallback : swv / sw;
    double a21 = a12, a31 = a13, a32 = a23;
    double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                 a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return fallback;
    double inv = 1.0 / fabs(det);
    return ((a22 * a33 - a23 * a32) * fw + (a13 * a32 - a12 * a33) * f1w + (a12 * a23 - a13 * a22) * f2w) * inv;
}

static double w_sig(const OMesh* m, const OField* f, const OStep* s, int slot, double xp, double yp, double z,
                    int node) {
    double alpha = stage_alpha(s, slot);
    if (s->w_code >= 2) return w_sig_ring(m, f, s, slot, alpha, xp, yp, z, node);
    if (s->w_code == 0) return w_sig_linear(m, f, alpha, z, node, col_H(m, f, s, node, slot), s->td);
    int verts[4];
    double wts[4];
    int nv = bary_locate(m, xp, yp, node, verts, wts);
    if (nv == 0) {
        double H = col_H(m, f, s, node, slot);
        double zc = z < H ? z : H;
        return w_sig_linear(m, f, alpha, zc, node, H, s->td);
    }
    double Hp = 0.0;
    for (int v = 0; v < nv; ++v) Hp += wts[v] * col_H(m, f, s, verts[v], slot);
    double fr = sigma_frac(z, Hp);
    double acc = 0.0;
    for (int v = 0; v < nv; ++v) {
        double Hv = col_H(m, f, s, verts[v], slot);
        acc += wts[v] * w_sig_linear(m, f, alpha, fr * Hv, verts[v], Hv, s->td);
    }
    return acc;
}

/* vertical_sigma.py:73-109 find_layer_sigma in the particle's column
 * (floored at Dmin, :135-144) */
static int find_layer_sig(const OMesh* m, double z, double H, double Dmin) {
    if (H < Dmin) H = Dmin;
    int K = m->K;
    const double* sg = m->sigma;
    if (K < 2) return 0;
    if (z <= (1.0 - sg[0]) * H) return 0;
    if (z >= (1.0 - sg[K - 1]) * H) return K - 2;
    for (int k = 0; k < K - 1; ++k)
        if (z < (1.0 - sg[k + 1]) * H) return k;
    return K - 2;
}

/* vertical_sigma.py:236-255 the clamp in the particle's column */
static double clamp_sig(double z, double H, const OStep* s) {
    if (H < s->Dmin) H = s->Dmin;
    if (z < 0.0) z = 0.0;
    double bottom = H - s->z0b_min;
    if (bottom < 0.0) bottom = 0.0;
    if (z > bottom) z = bottom;
    return z;
}

/* integrators.py:1351-1376 _sigma_frac_for_uv (a NaN stays NaN) */
static double sfrac_uv(double z, double H) {
    double fr = z / H;
    if (fr < 0.0) fr = 0.0;
    if (fr > 1.0) fr = 1.0;
    return fr;
}

/* u/v of a sigma stage: the layer in the particle's column, or the
 * depth-linear rule read in s (vertical_uv.py:196-211) */
static int sig_stage_uv(const OMesh* m, const OField* f, const OStep* s, double xp, double yp, int nn, double z,
                        double H, double alpha, double* U, double* V) {
    if (s->uv_dl) return interp_uv_dl(m, f, xp, yp, nn, sfrac_uv(z, H), s->td, alpha, U, V);
    return interp_uv(m, f, xp, yp, nn, s->td, find_layer_sig(m, z, H, s->Dmin), alpha, U, V);
}

/* One particle of the sigma step: integrators.py:4997-5147 (Euler),
 * :5380-5608 (RK2, unfused), :5760-6011 (RK4, unfused), sigma branches;
 * the split kick keeps s = z / H_p into the kicked column (:783-803). */
static void step_sigma(const OMesh* m, const OField* f, const OStep* s, int64_t i, double* lon, double* lat,
                       double* z, int* status, int* nn, int8_t* fr, double* U, double* V, double* W,
                       const int64_t* pid, int32_t* elem) {
    double lon0 = lon[i], lat0 = lat[i], zp = z[i], dt = s->dt;
    int pre_nn = nn[i], st = ALIVE, nno, _r;
    int8_t frr = fr[i];
    double ln = lon0, lt = lat0, zn = zp;
    int node_i = anchor(m, lon0, lat0);
    nno = node_i;
    const int walk = elem != NULL;
    const int e1 = walk ? walk_locate(m, lon0, lat0, elem[i], node_i) : -1;
    int e_last = e1, e_out = e1;
#define LOC(x, y, from, n) (walk ? walk_locate(m, (x), (y), (from), (n)) : -1)
    double H1 = sigma_H(m, f, s, 0, lon0, lat0, node_i);
    double U1, V1;
    int ok = STAGE(e1, sig_stage_uv(m, f, s, lon0, lat0, node_i, zp, H1, s->ak[0], &U1, &V1));
    double W1 = w_sig(m, f, s, 0, lon0, lat0, zp, node_i);
    U[i] = U1; V[i] = V1; W[i] = W1;
    double a = lon0, b = lat0, s_new = 0.0;
    if (ok) {
        if (s->scheme == 0) {
            a = wrap180(lon0 + dt * U1 / z0_of(lat0));
            b = clat(lat0 + dt * V1 / SLM);
            s_new = (zp + W1 * dt) / H1;
        } else if (s->scheme == 1) {
            double lm = wrap180(lon0 + 0.5 * dt * U1 / z0_of(lat0));
            double tm = clat(lat0 + 0.5 * dt * V1 / SLM);
            double s_mid = (zp + W1 * 0.5 * dt) / H1;
            int nm = anchor(m, lm, tm);
            int em = LOC(lm, tm, e1, nm);
            e_last = em;
            double H2 = sigma_H(m, f, s, 1, lm, tm, nm);
            double zm = s_mid * H2;
            double U2, V2;
            if (!STAGE(em, sig_stage_uv(m, f, s, lm, tm, nm, zm, H2, s->ak[1], &U2, &V2))) ok = 0;
            else {
                double W2 = w_sig(m, f, s, 1, lm, tm, zm, nm);
                a = wrap180(lon0 + dt * U2 / z0_of(tm));
                b = clat(lat0 + dt * V2 / SLM);
                s_new = zp / H1 + dt * W2 / H2;
            }
        } else {
            double dl1 = dt * U1 / z0_of(lat0), dd1 = dt * V1 / SLM;
            double s0 = zp / H1, f1 = W1 / H1;
            double l2 = wrap180(lon0 + 0.5 * dl1), t2 = clat(lat0 + 0.5 * dd1);
            int n2 = anchor(m, l2, t2), e2 = LOC(l2, t2, e1, n2);
            double H2 = sigma_H(m, f, s, 1, l2, t2, n2);
            double z2 = (s0 + 0.5 * dt * f1) * H2;
            double U2, V2, U3, V3, U4, V4;
            if (!STAGE(e2, sig_stage_uv(m, f, s, l2, t2, n2, z2, H2, s->ak[1], &U2, &V2))) ok = 0;
            else {
                double W2 = w_sig(m, f, s, 1, l2, t2, z2, n2);
                double dl2 = dt * U2 / z0_of(t2), dd2 = dt * V2 / SLM, f2 = W2 / H2;
                double l3 = wrap180(lon0 + 0.5 * dl2), t3 = clat(lat0 + 0.5 * dd2);
                int n3 = anchor(m, l3, t3), e3 = LOC(l3, t3, e2, n3);
                double H3 = sigma_H(m, f, s, 2, l3, t3, n3);
                double z3 = (s0 + 0.5 * dt * f2) * H3;
                if (!STAGE(e3, sig_stage_uv(m, f, s, l3, t3, n3, z3, H3, s->ak[2], &U3, &V3))) ok = 0;
                else {
                    double W3 = w_sig(m, f, s, 2, l3, t3, z3, n3);
                    double dl3 = dt * U3 / z0_of(t3), dd3 = dt * V3 / SLM, f3 = W3 / H3;
                    double l4 = wrap180(lon0 + dl3), t4 = clat(lat0 + dd3);
                    int n4 = anchor(m, l4, t4), e4 = LOC(l4, t4, e3, n4);
                    e_last = e4;
                    double H4 = sigma_H(m, f, s, 3, l4, t4, n4);
                    double z4 = (s0 + dt * f3) * H4;
                    if (!STAGE(e4, sig_stage_uv(m, f, s, l4, t4, n4, z4, H4, s->ak[3], &U4, &V4))) ok = 0;
                    else {
                        double W4 = w_sig(m, f, s, 3, l4, t4, z4, n4);
                        double dl4 = dt * U4 / z0_of(t4), dd4 = dt * V4 / SLM, f4 = W4 / H4;
                        double dl = (dl1 + 2.0 * dl2 + 2.0 * dl3 + dl4) / 6.0;
                        double dd = (dd1 + 2.0 * dd2 + 2.0 * dd3 + dd4) / 6.0;
                        a = wrap180(lon0 + dl);
                        b = clat(lat0 + dd);
                        s_new = s0 + dt * (f1 + 2.0 * f2 + 2.0 * f3 + f4) / 6.0;
                    }
                }
            }
        }
    }
    if (!ok) { st = OUTSIDE; frr = 1; }
    else {
        int nw = anchor(m, a, b);
        int ein = walk ? walk_locate(m, a, b, e_last, nw) : contain_local(m, a, b, nw);
        if (ein < 0) { st = OUTSIDE; frr = 2; }
        else {
            double He = sigma_H(m, f, s, 4, a, b, nw);
            ln = a; lt = b; nno = nw; e_out = ein;
            zn = clamp_sig(s_new * He, He, s);
        }
    }
#undef LOC
    if (s->kick && st == ALIVE) {
        double plon = ln, plat = lt;
        int pnn = nno;
        kick(m, s, pid ? pid[i] : i, lon0, lat0, zp, pre_nn, &ln, &lt, &zn, &st, &nno, &frr, 0);
        if (st == ALIVE) {
            double Hpost = sigma_H(m, f, s, 4, plon, plat, pnn);
            double Hk = sigma_H(m, f, s, 4, ln, lt, nno);
            zn = clamp_sig(zn / Hpost * Hk, Hk, s);
        }
    }
    if (s->az_on && st == ALIVE) az_kick_sigma(s, pid ? pid[i] : i, sigma_H(m, f, s, 4, ln, lt, nno), &zn);
    lon[i] = ln; lat[i] = lt; z[i] = zn;
    status[i] = st; nn[i] = nno; fr[i] = frr;
    if (walk) elem[i] = e_out;
}


static void step_one(const OMesh* m, const OField* f, const OStep* s, int64_t i, double* lon, double* lat, double* z,
                     int* status, int* nn, int8_t* fr, double* U, double* V, double* W, const int64_t* pid,
                     int32_t* elem) {
    if (m->cg && s->dims == 3) {
        step_cgrid3d(m, f, s, i, lon, lat, z, status, nn, fr, U, V, W);
        return;
    }
    if (status[i] != ALIVE) {
        U[i] = 0.0; V[i] = 0.0;
        if (W) W[i] = 0.0;
        return;
    }
    if (m->sig && s->dims == 3) {
        step_sigma(m, f, s, i, lon, lat, z, status, nn, fr, U, V, W, pid, elem);
        return;
    }
    double lon0 = lon[i], lat0 = lat[i], zp = z ? z[i] : 0.0, dt = s->dt, td = s->td;
    int pre_nn = nn[i], st = ALIVE, nno, _r;
    int8_t frr = fr[i];
    double ln = lon0, lt = lat0, zn = zp;
    int node_i = anchor(m, lon0, lat0);
    nno = node_i;
    const int walk = elem != NULL;
    const int e1 = walk ? walk_locate(m, lon0, lat0, elem[i], node_i) : -1;
    int e_last = e1, e_out = e1;
#define LOC(x, y, from, n) (walk ? walk_locate(m, (x), (y), (from), (n)) : -1)
    int ok = 1;
    if (s->dims == 2) {
        double U1, V1;
        int ok1 = STAGE(e1, uv2(m, f, lon0, lat0, node_i, td, s->ak[0], &U1, &V1));
        U[i] = U1; V[i] = V1;
        if (!ok1) { ok = 0; }
        else if (s->scheme == 0) {
            ln = wrap180(lon0 + dt * U1 / z0_of(lat0));
            lt = clat(lat0 + dt * V1 / SLM);
        } else if (s->scheme == 1) {
            double lm = wrap180(lon0 + 0.5 * dt * U1 / z0_of(lat0));
            double tm = clat(lat0 + 0.5 * dt * V1 / SLM);
            int nm = anchor(m, lm, tm);
            int em = LOC(lm, tm, e1, nm);
            e_last = em;
            double U2, V2;
            if (!STAGE(em, uv2(m, f, lm, tm, nm, td, s->ak[1], &U2, &V2))) ok = 0;
            else { ln = wrap180(lon0 + dt * U2 / z0_of(tm)); lt = clat(lat0 + dt * V2 / SLM); }
        } else {
            double dl1 = dt * U1 / z0_of(lat0), dt1 = dt * V1 / SLM;
            double l2 = wrap180(lon0 + 0.5 * dl1), t2 = clat(lat0 + 0.5 * dt1);
            double U2, V2, U3, V3, U4, V4;
            int n2 = anchor(m, l2, t2), e2 = LOC(l2, t2, e1, n2);
            if (!STAGE(e2, uv2(m, f, l2, t2, n2, td, s->ak[1], &U2, &V2))) ok = 0;
            else {
                double dl2 = dt * U2 / z0_of(t2), dt2 = dt * V2 / SLM;
                double l3 = wrap180(lon0 + 0.5 * dl2), t3 = clat(lat0 + 0.5 * dt2);
                int n3 = anchor(m, l3, t3), e3 = LOC(l3, t3, e2, n3);
                if (!STAGE(e3, uv2(m, f, l3, t3, n3, td, s->ak[2], &U3, &V3))) ok = 0;
                else {
                    double dl3 = dt * U3 / z0_of(t3), dt3 = dt * V3 / SLM;
                    double l4 = wrap180(lon0 + dl3), t4 = clat(lat0 + dt3);
                    int n4 = anchor(m, l4, t4), e4 = LOC(l4, t4, e3, n4);
                    e_last = e4;
                    if (!STAGE(e4, uv2(m, f, l4, t4, n4, td, s->ak[3], &U4, &V4))) ok = 0;
                    else {
                        double dl4 = dt * U4 / z0_of(t4), dt4 = dt * V4 / SLM;
                        double dl = (dl1 + 2.0 * dl2 + 2.0 * dl3 + dl4) / 6.0;
                        double dd = (dt1 + 2.0 * dt2 + 2.0 * dt3 + dt4) / 6.0;
                        ln = wrap180(lon0 + dl);
                        lt = clat(lat0 + dd);
                    }
                }
            }
        }
        if (!ok) { st = OUTSIDE; frr = 1; ln = lon0; lt = lat0; }
        else {
            int nw = anchor(m, ln, lt);
            int ein = walk ? walk_locate(m, ln, lt, e_last, nw) : contain_local(m, ln, lt, nw);
            if (ein < 0) { st = OUTSIDE; frr = 2; ln = lon0; lt = lat0; }
            else { nno = nw; e_out = ein; }
        }
    } else if (s->scheme != 1) {
        /* 3-D Euler (integrators.py:4997-5147) and RK4 (:5760-6011): the
         * unfused multi-pass paths restated per particle -- batch exact anchor
         * per stage, layer at the stage depth, stage fields blended per vertex
         * (the whole-field lerps of _make_stage_vels, :1187-1237), W at the
         * stage position, failure reverts to the start with the start anchor. */
        double U1, V1;
        int ok1 = STAGE(e1, stage_uv(m, f, s, lon0, lat0, node_i, zp, s->ak[0], &U1, &V1));
        double W1 = w_stage(m, f, s->w_code, s->ak[0], lon0, lat0, zp, node_i, td);
        U[i] = U1; V[i] = V1; W[i] = W1;
        double a = lon0, b = lat0, c = zp;
        if (!ok1) ok = 0;
        else if (s->scheme == 0) {
            a = wrap180(lon0 + dt * U1 / z0_of(lat0));
            b = clat(lat0 + dt * V1 / SLM);
            c = zp + W1 * dt;
        } else {
            double dl1 = dt * U1 / z0_of(lat0), dd1 = dt * V1 / SLM, dz1 = dt * W1;
            double l2 = wrap180(lon0 + 0.5 * dl1), t2 = clat(lat0 + 0.5 * dd1), z2 = zp + 0.5 * dz1;
            int n2 = anchor(m, l2, t2), e2 = LOC(l2, t2, e1, n2);
            double U2, V2, U3, V3, U4, V4;
            if (!STAGE(e2, stage_uv(m, f, s, l2, t2, n2, z2, s->ak[1], &U2, &V2))) ok = 0;
            else {
                double W2 = w_stage(m, f, s->w_code, s->ak[1], l2, t2, z2, n2, td);
                double dl2 = dt * U2 / z0_of(t2), dd2 = dt * V2 / SLM, dz2 = dt * W2;
                double l3 = wrap180(lon0 + 0.5 * dl2), t3 = clat(lat0 + 0.5 * dd2), z3 = zp + 0.5 * dz2;
                int n3 = anchor(m, l3, t3), e3 = LOC(l3, t3, e2, n3);
                if (!STAGE(e3, stage_uv(m, f, s, l3, t3, n3, z3, s->ak[2], &U3, &V3))) ok = 0;
                else {
                    double W3 = w_stage(m, f, s->w_code, s->ak[2], l3, t3, z3, n3, td);
                    double dl3 = dt * U3 / z0_of(t3), dd3 = dt * V3 / SLM, dz3 = dt * W3;
                    double l4 = wrap180(lon0 + dl3), t4 = clat(lat0 + dd3), z4 = zp + dz3;
                    int n4 = anchor(m, l4, t4), e4 = LOC(l4, t4, e3, n4);
                    e_last = e4;
                    if (!STAGE(e4, stage_uv(m, f, s, l4, t4, n4, z4, s->ak[3], &U4, &V4))) ok = 0;
                    else {
                        double W4 = w_stage(m, f, s->w_code, s->ak[3], l4, t4, z4, n4, td);
                        double dl4 = dt * U4 / z0_of(t4), dd4 = dt * V4 / SLM, dz4 = dt * W4;
                        double dl = (dl1 + 2.0 * dl2 + 2.0 * dl3 + dl4) / 6.0;
                        double dd = (dd1 + 2.0 * dd2 + 2.0 * dd3 + dd4) / 6.0;
                        double dz = (dz1 + 2.0 * dz2 + 2.0 * dz3 + dz4) / 6.0;
                        a = wrap180(lon0 + dl);
                        b = clat(lat0 + dd);
                        c = zp + dz;
                    }
                }
            }
        }
        if (!ok) { st = OUTSIDE; frr = 1; }
        else {
            int nw = anchor(m, a, b);
            int ein = walk ? walk_locate(m, a, b, e_last, nw) : contain_local(m, a, b, nw);
            if (ein < 0) { st = OUTSIDE; frr = 2; }
            else {
                if (c < m->zlev[0]) c = m->zlev[0];
                if (c > m->depth[nw]) c = m->depth[nw];
                ln = a; lt = b; zn = c; nno = nw; e_out = ein;
            }
        }
    } else {
        double U1, V1;
        int ok1 = STAGE(e1, stage_uv(m, f, s, lon0, lat0, node_i, zp, s->ak[0], &U1, &V1));
        double W1 = w_stage(m, f, s->w_code, s->ak[0], lon0, lat0, zp, node_i, td);
        U[i] = U1; V[i] = V1; W[i] = W1;
        if (!ok1) { st = OUTSIDE; frr = 1; }
        else {
            double lm = wrap180(lon0 + 0.5 * dt * U1 / z0_of(lat0));
            double tm = clat(lat0 + 0.5 * dt * V1 / SLM);
            double zm = zp + W1 * 0.5 * dt;
            int nm = anchor(m, lm, tm);
            int em = LOC(lm, tm, e1, nm);
            e_last = em;
            double U2, V2;
            if (!STAGE(em, stage_uv(m, f, s, lm, tm, nm, zm, s->ak[1], &U2, &V2))) { st = OUTSIDE; frr = 1; }
            else {
                double W2 = w_stage(m, f, s->w_code, s->ak[1], lm, tm, zm, nm, td);
                double a = wrap180(lon0 + dt * U2 / z0_of(tm));
                double b = clat(lat0 + dt * V2 / SLM);
                double c = zp + W2 * dt;
                int nw = anchor(m, a, b);
                int ein = walk ? walk_locate(m, a, b, e_last, nw) : contain_local(m, a, b, nw);
                if (ein < 0) { st = OUTSIDE; frr = 2; }
                else {
                    if (c < m->zlev[0]) c = m->zlev[0];
                    if (c > m->depth[nw]) c = m->depth[nw];
                    ln = a; lt = b; zn = c; nno = nw; e_out = ein;
                }
            }
        }
    }
#undef LOC
    if (s->kick && st == ALIVE)
        kick(m, s, pid ? pid[i] : i, lon0, lat0, zp, pre_nn, &ln, &lt, &zn, &st, &nno, &frr, s->dims == 3);
    if (s->az_on && st == ALIVE && s->dims == 3) az_kick(m, f, s, pid ? pid[i] : i, nno, &zn);
    lon[i] = ln; lat[i] = lt;
    if (z) z[i] = zn;
    status[i] = st; nn[i] = nno; fr[i] = frr;
    if (walk) elem[i] = e_out;
}


/* mesh.py:2593-2712 for a batch: the walk from start[i] (-1: none) */
typedef struct { const OMesh* m; const double *lon, *lat; const int* start; const int* nn; int* out; } WCtx;
static void walk_body(void* ctx, int64_t i) {
    WCtx* c = (WCtx*)ctx;
    c->out[i] = walk_locate(c->m, c->lon[i], c->lat[i], c->start[i], c->nn[i]);
}

/* ---- a small dynamic parallel-for over particles (pthreads) ---------- */

typedef void (*orc_body)(void* ctx, int64_t i);
typedef struct {
    orc_body fn;
    void* ctx;
    int64_t n, chunk;
    int64_t next;
    pthread_mutex_t mu;
} orc_pool;

static int g_threads = 0;

int orc_set_threads(int n) { g_threads = n; return 0; }

int orc_get_threads(void) {
    if (g_threads > 0) return g_threads;
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static void* orc_worker(void* arg) {
    orc_pool* p = (orc_pool*)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        int64_t s = p->next;
        p->next += p->chunk;
        pthread_mutex_unlock(&p->mu);
        if (s >= p->n) break;
        int64_t e = s + p->chunk < p->n ? s + p->chunk : p->n;
        for (int64_t i = s; i < e; ++i) p->fn(p->ctx, i);
    }
    return NULL;
}

static void par_for(int64_t n, orc_body fn, void* ctx) {
    int nt = orc_get_threads();
    if (nt > 256) nt = 256;
    orc_pool p;
    p.fn = fn; p.ctx = ctx; p.n = n; p.chunk = 256; p.next = 0;
    pthread_mutex_init(&p.mu, NULL);
    if (nt <= 1 || n < 1024) {
        orc_worker(&p);
    } else {
        pthread_t th[256];
        for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, orc_worker, &p);
        for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
    }
    pthread_mutex_destroy(&p.mu);
}

/* ---- exported entry points (ctypes) ---------------------------------- */

typedef struct {
    int64_t N, E;
    int max_v, max_conn;
    const double *lon, *lat, *depth, *xyz, *zlev;
    const int32_t *en, *n2e, *n2e_cnt, *gh_off, *gh_ids;
    double cell, lon_min, lat_min, r_earth;
    int nx, ny, wrap, far_rows, exact, K;
    const double *dl_p, *dl_bed;
    const int32_t* dl_last;
    int dl_M;
    const int32_t* enb;
    const double* sigma;
    int sig;
    int cg;                        /* 1: a NEMO C-grid mesh (readers/nemo/_mesh.py build_nemo_cgrid_mesh) */
    const int32_t* cg_corners;     /* (E, 4) F-point corners SW, SE, NE, NW */
    const int64_t* cg_ji;          /* (E, 2) T-cell (j, i) */
    const int32_t* cg_nlev;        /* (E) wet levels (0: the dry ring) */
    const int32_t* cg_nlev_r;      /* (ny*nx) wet levels per column */
    int cg_nx, cg_K, cg_shrunk, cg_has_e;
    int64_t cg_nynx;
    const double *cg_e2u, *cg_e1v, *cg_area, *cg_zw, *cg_e3b, *cg_e3u, *cg_e3v;
    const int32_t *cg_kbu, *cg_kbv;
    const double *ec_lon, *ec_lat;
} orc_mesh;

typedef struct {
    const void *ua, *va, *wa, *ub, *vb, *wb, *ut, *vt, *wt;
    int f32;
    double alpha0;
    int64_t n;
    const void *aza, *azb;
    const double *etaa, *etab, *etat;
    int pchip;
    const void *ud, *vd, *wd;
    const double* etad;
    double pt[4];
    int lsq;
} orc_field;

typedef struct {
    int scheme, dims, w_code, kick;
    double dt, td, ak[4], kh_x, kh_y;
    uint64_t seed, real_id, step_i, pid_offset;
    int uv_dl;
    int az_on, az_field;
    double az_const;
    double Dmin, z0b_min, alpha_end;
    const double *eta_s, *eta_e;
    int sig_steady;
} orc_step_args;

typedef struct {
    const OMesh* m; const OField* f; const OStep* s;
    double *lon, *lat, *z; int *status, *nn; int8_t* fr; double *U, *V, *W; const int64_t* pid;
    int32_t* elem;
} StepCtx;

static void step_body(void* ctx, int64_t i) {
    StepCtx* c = (StepCtx*)ctx;
    step_one(c->m, c->f, c->s, i, c->lon, c->lat, c->z, c->status, c->nn, c->fr, c->U, c->V, c->W, c->pid,
             c->elem);
}

typedef struct { const OMesh* m; const double *lon, *lat; const int* nn; int* out; } QCtx;
static void near_body(void* ctx, int64_t i) { QCtx* c = (QCtx*)ctx; c->out[i] = anchor(c->m, c->lon[i], c->lat[i]); }
static void cont_body(void* ctx, int64_t i) { QCtx* c = (QCtx*)ctx; c->out[i] = contain_local(c->m, c->lon[i], c->lat[i], c->nn[i]); }

int orc_step(const orc_mesh* mm, const orc_field* ff, const orc_step_args* ss, int64_t P, double* lon, double* lat,
             double* z, int* status, int* nn, int8_t* fr, double* U, double* V, double* W, const int64_t* pid,
             const int* release_step, int64_t global_step, int32_t* elem) {
    const OMesh* m = (const OMesh*)mm;
    const OField* f = (const OField*)ff;
    const OStep* s = (const OStep*)ss;
    if (release_step && global_step >= 0)
        for (int64_t i = 0; i < P; ++i)
            if (status[i] == NOT_RELEASED && global_step >= release_step[i]) status[i] = ALIVE;
    StepCtx c = {m, f, s, lon, lat, z, status, nn, fr, U, V, W, pid, elem};
    par_for(P, step_body, &c);
    return 0;
}

int orc_walk(const orc_mesh* mm, int64_t P, const double* lon, const double* lat, const int* start, const int* nn,
             int* out) {
    WCtx c = {(const OMesh*)mm, lon, lat, start, nn, out};
    par_for(P, walk_body, &c);
    return 0;
}

int orc_find_nearest(const orc_mesh* mm, int64_t P, const double* lon, const double* lat, int* out) {
    const OMesh* m = (const OMesh*)mm;
    QCtx c = {m, lon, lat, NULL, out};
    par_for(P, near_body, &c);
    return 0;
}

/* mesh.py:353-380 _gh_rect_sum over the (ny+1) x (nx+1) prefix table cum */
static int64_t rect_sum(const int32_t* cum, int nx, int ny, int wrap, int ci, int cj, int rx, int ry) {
    int64_t W = nx + 1;
    int j0 = cj - ry < 0 ? 0 : cj - ry;
    int j1 = cj + ry + 1 > ny ? ny : cj + ry + 1;
#define CUM(j, i) ((int64_t)cum[(int64_t)(j) * W + (i)])
    if (wrap && 2 * rx + 1 >= nx) return CUM(j1, nx) - CUM(j0, nx);
    int i0 = ci - rx, i1 = ci + rx + 1;
    if (wrap) {
        if (i0 < 0)
            return (CUM(j1, i1) - CUM(j0, i1)) + (CUM(j1, nx) - CUM(j0, nx)) - (CUM(j1, i0 + nx) - CUM(j0, i0 + nx));
        if (i1 > nx)
            return (CUM(j1, nx) - CUM(j0, nx)) - (CUM(j1, i0) - CUM(j0, i0)) + (CUM(j1, i1 - nx) - CUM(j0, i1 - nx));
    } else {
        if (i0 < 0) i0 = 0;
        if (i1 > nx) i1 = nx;
    }
    return (CUM(j1, i1) - CUM(j0, i1)) - (CUM(j1, i0) - CUM(j0, i0));
#undef CUM
}

/* mesh.py:384-461 _gh_sample_stats for one candidate grid (cell, lon_min,
 * lat_min, nx, ny, wrap over the mesh's nodes; cum its prefix table) at P
 * samples with their nearest nodes nn.  Serial: a test-size checker. */
int orc_cell_stats(const orc_mesh* mm, const int32_t* cum, double cell, double lon_min, double lat_min, int nx,
                   int ny, int wrap, int64_t P, const double* lon, const double* lat, const int32_t* nn,
                   int64_t* occ_out, double* cost_out, int8_t* unprov_out, int8_t* approx_out) {
    OMesh g = *(const OMesh*)mm;
    g.cell = cell; g.lon_min = lon_min; g.lat_min = lat_min; g.nx = nx; g.ny = ny; g.wrap = wrap;
    for (int64_t i = 0; i < P; ++i) {
        int ci, cj, cin, cjn;
        cell_of(&g, lon[i], lat[i], &ci, &cj);
        int64_t occ = rect_sum(cum, nx, ny, wrap, ci, cj, 1, 1);
        occ_out[i] = occ;
        cell_of(&g, g.lon[nn[i]], g.lat[nn[i]], &cin, &cjn);
        int di = cin - ci < 0 ? ci - cin : cin - ci;
        if (wrap && nx - di < di) di = nx - di;
        int dj = cjn - cj < 0 ? cj - cjn : cjn - cj;
        approx_out[i] = (di > 1 || dj > 1) ? 1 : 0;
        double theta, ext;
        cap_extents(lon[i], lat[i], g.lon[nn[i]], g.lat[nn[i]], &theta, &ext);
        int provable = occ > 0 && approx_out[i] == 0;
        if (provable) provable = provable_rect(&g, lon[i], lat[i], nn[i], 1, 1) == 0;
        if (provable) {
            cost_out[i] = (double)occ + 9.0 * 1.0 + 20.0;
            unprov_out[i] = 0;
            continue;
        }
        int ry = (int)ceil(theta / cell);
        if (ry < 1) ry = 1;
        if (ry > ny) ry = ny;
        int rx;
        if (ext >= 1.0e29) {
            rx = nx;
        } else {
            rx = (int)ceil(ext / cell);
            if (rx < 1) rx = 1;
        }
        int64_t cells, iters;
        if (rx * 2 + 1 >= nx) {
            rx = nx;
            cells = 9 + 2 * (int64_t)ry;
            iters = ry;
        } else {
            cells = 9 + (int64_t)rx * (2 * (int64_t)ry + 1) + 2 * (int64_t)ry;
            iters = rx > ry ? rx : ry;
        }
        cost_out[i] = ((double)rect_sum(cum, nx, ny, wrap, ci, cj, rx, ry) + (double)cells * 1.0) +
                      (double)(iters + 1) * 20.0;
        unprov_out[i] = 1;
    }
    return 0;
}

int orc_contain(const orc_mesh* mm, int64_t P, const double* lon, const double* lat, const int* nn, int* out) {
    const OMesh* m = (const OMesh*)mm;
    QCtx c = {m, lon, lat, nn, out};
    par_for(P, cont_body, &c);
    return 0;
}

/* tracking.py:199-364 _apply_beaching_hook with beaching.py:95-181
 * evaluate_beaching, over all particles in index order (serial: the
 * reference's stochastic loops are serial too). */
typedef struct {
    int use_depth, use_coastal, use_stochastic, on_failure;
    int resuspension, min_wet_steps;
    double depth_min, zone_depth, rewet_hysteresis, p_beach, p_resusp;
    uint64_t seed, real_id, step_i, pid_offset;
} orc_beach_args;

static double u01(uint64_t seed, uint64_t real_id, uint64_t pid, uint64_t step, uint64_t comp) {
    uint64_t h = orc_key_hash(seed, real_id, pid, step, comp);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

/* eta (N): the payload's free surface when use_eta, else NULL; dry (N): the
 * dry-mask variable's surface layer, else NULL (tracking.py:236-327). */
int orc_beach(const orc_mesh* mm, const orc_beach_args* a, const unsigned char* coastal, int64_t P,
              const double* lon, const double* lat, int* status, const int* prev, int* nn, int8_t* fr,
              int* wet, const double* eta, const double* dry) {
    const OMesh* m = (const OMesh*)mm;
    int need_topo = a->use_coastal || a->use_stochastic;
    int any_beached = 0;
    /* stale anchors of newly failed particles, containing elements, remap */
    int* cont = (int*)malloc(sizeof(int) * (P > 0 ? P : 1));
    for (int64_t i = 0; i < P; ++i) {
        int newly = status[i] == OUTSIDE && prev[i] == ALIVE;
        if (newly && nn[i] < 0) nn[i] = anchor(m, lon[i], lat[i]);
        cont[i] = -1;
        if (need_topo && (status[i] == ALIVE || status[i] == 2 || newly)) {
            int a0 = nn[i] < 0 ? (int)(nn[i] + m->N) : nn[i];
            cont[i] = contain_local(m, lon[i], lat[i], a0);
        }
        if (a->on_failure && newly) {
            double hf = INFINITY;
            if (nn[i] >= 0) { hf = m->depth[nn[i]]; if (eta) hf = hf + eta[nn[i]]; }
            int context = hf < a->zone_depth;
            if (need_topo && cont[i] >= 0 && coastal[cont[i]]) context = 1;
            if (context) { status[i] = 2; fr[i] = 0; }
        }
    }
    for (int64_t i = 0; i < P; ++i) any_beached |= status[i] == 2;
    double rewet_level = a->depth_min + a->rewet_hysteresis;
    for (int64_t i = 0; i < P; ++i) {
        int alive = status[i] == ALIVE, beached = status[i] == 2;
        double h = INFINITY;
        if (nn[i] >= 0) { h = m->depth[nn[i]]; if (eta) h = h + eta[nn[i]]; }
        int masked = dry && nn[i] >= 0 && dry[nn[i]] > 0.5;
        int cc = need_topo && cont[i] >= 0 && coastal[cont[i]];
        uint64_t key = (uint64_t)i + a->pid_offset;
        int to_beach = 0;
        if (a->use_depth && (h < a->depth_min || masked)) to_beach = 1;
        if (a->use_coastal && cc) to_beach = 1;
        if (a->use_stochastic && alive) {
            int in_zone = h < a->zone_depth || cc;
            if (in_zone && u01(a->seed, a->real_id, key, a->step_i, 10) < a->p_beach) to_beach = 1;
        }
        to_beach = to_beach && alive;
        int ws = wet[i], to_release = 0;
        if (a->resuspension != 0 && any_beached && beached) {
            int rewet = h > rewet_level && nn[i] >= 0 && !masked;
            ws = rewet ? ws + 1 : 0;
            if (a->resuspension == 1 || a->resuspension == 3) to_release = to_release || ws >= a->min_wet_steps;
            if ((a->resuspension == 2 || a->resuspension == 3) && rewet &&
                u01(a->seed, a->real_id, key, a->step_i, 11) < a->p_resusp)
                to_release = 1;
        }
        if (to_release) ws = 0;
        if (!beached) ws = 0;
        if (to_beach) status[i] = 2;
        if (to_release) { status[i] = ALIVE; fr[i] = 0; }
        wet[i] = ws;
    }
    free(cont);
    return 0;
}

int orc_normals(int64_t P, uint64_t seed, uint64_t real_id, uint64_t step, uint64_t pid_offset, uint64_t comp,
                double* g) {
    for (int64_t i = 0; i < P; ++i) orc_normal_pair(seed, real_id, (uint64_t)i + pid_offset, step, comp, g + 2 * i);
    return 0;
}

int orc_node_xyz(int64_t n, const double* lon, const double* lat, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        double cl;
        qxyz(lon[i], lat[i], out + 3 * i, out + 3 * i + 1, out + 3 * i + 2, &cl);
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * Scalar field sampling at particle positions (numerics/sampling.py).
 * ------------------------------------------------------------------------ */
#define S_NEAREST 0
#define S_LEASTSQ 1
#define S_BARYCENTRIC 2
#define S_IDW 3
/* sampling.py:82-380 _combine_horizontal */
static double combine_horizontal(const OMesh* m, const double* vals, const int32_t* buf, int cnt, double lon_p,
                                 double lat_p, int nn, int method) {
    double fallback = vals[0];
    if (method == S_NEAREST) return fallback;
    if (method == S_IDW) {
        double z0 = cos(lat_p * DEG2RAD) * SLM;
        if (z0 < 1.0) z0 = 1.0;
        double sw = 0.0, swv = 0.0;
        for (int i = 0; i < cnt; ++i) {
            int nd = buf[i];
            double dx = wrap180(m->lon[nd] - lon_p) * z0;
            double dy = (m->lat[nd] - lat_p) * SLM;
            double d2 = dx * dx + dy * dy;
            if (d2 < 1e-12) return vals[i];
            if (!isfinite(vals[i])) continue;
            double w = 1.0 / d2;
            sw += w;
            swv += w * vals[i];
        }
        if (sw < 1e-30) return fallback;
        return swv / sw;
    }
    if (method == S_BARYCENTRIC) {
        int ne = m->n2e_cnt[nn];
        for (int k = 0; k < ne; ++k) {
            int e = m->n2e[(int64_t)nn * m->max_conn + k];
            if (e < 0) continue;
            int verts[4], nv = 0;
            for (int v = 0; v < m->max_v; ++v) {
                int nd = m->en[(int64_t)e * m->max_v + v];
                if (nd < 0) continue;
                if (nv > 0 && nd == verts[0]) continue;
                verts[nv++] = nd;
            }
            if (nv < 3) continue;
            double ln[4], vx[4], vy[4];
            for (int v = 0; v < nv; ++v) ln[v] = m->lon[verts[v]];
            double lon0 = seam_lon0(ln, nv);
            double lat0 = 0.0;
            for (int v = 0; v < nv; ++v) lat0 += m->lat[verts[v]];
            lat0 /= nv;
            double cl = cos(lat0 * DEG2RAD);
            for (int v = 0; v < nv; ++v) {
                vx[v] = wrap180(m->lon[verts[v]] - lon0) * DEG2RAD * R_STD * cl;
                vy[v] = (m->lat[verts[v]] - lat0) * DEG2RAD * R_STD;
            }
            double px = wrap180(lon_p - lon0) * DEG2RAD * R_STD * cl;
            double py = (lat_p - lat0) * DEG2RAD * R_STD;
            for (int t = 0; t < nv - 2; ++t) {
                double ax = vx[0], ay = vy[0], bx = vx[t + 1], by = vy[t + 1], cx = vx[t + 2], cy = vy[t + 2];
                double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
                if (fabs(denom) < 1e-14) continue;
                double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
                double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
                double w3 = 1.0 - w1 - w2;
                if (!(w1 >= -1e-6 && w2 >= -1e-6 && w3 >= -1e-6)) continue;
                if (nv == 4) {
                    double wts[4], acc = 0.0;
                    polygon_weights(px, py, vx, vy, 4, wts);
                    for (int vi = 0; vi < 4; ++vi) {
                        double vv = vals[0];
                        int fnd = 0;
                        for (int j = 0; j < cnt; ++j)
                            if (buf[j] == verts[vi]) { vv = vals[j]; fnd = 1; break; }
                        if (!fnd || !isfinite(vv)) return fallback;
                        acc += wts[vi] * vv;
                    }
                    return acc;
                }
                int n0 = verts[0], n1 = verts[t + 1], n2 = verts[t + 2];
                double v0 = vals[0], v1 = vals[0], v2 = vals[0];
                int f0 = 0, f1 = 0, f2 = 0;
                for (int j = 0; j < cnt; ++j) {
                    if (buf[j] == n0) { v0 = vals[j]; f0 = 1; }
                    if (buf[j] == n1) { v1 = vals[j]; f1 = 1; }
                    if (buf[j] == n2) { v2 = vals[j]; f2 = 1; }
                }
                if (!(f0 && f1 && f2)) return fallback;
                if (!(isfinite(v0) && isfinite(v1) && isfinite(v2))) return fallback;
                return w1 * v0 + w2 * v1 + w3 * v2;
            }
        }
        return fallback;
    }
    if (method == S_LEASTSQ) {
        if (cnt < 3) return fallback;
        double z0 = cos(lat_p * DEG2RAD) * SLM;
        if (z0 < 1.0) z0 = 1.0;
        double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0, f0 = 0.0, f1 = 0.0, f2 = 0.0;
        int nfin = 0;
        for (int i = 0; i < cnt; ++i) {
            int nd = buf[i];
            double val = vals[i];
            if (!isfinite(val)) continue;
            nfin++;
            double ex = wrap180(m->lon[nd] - lon_p) * z0;
            double ey = (m->lat[nd] - lat_p) * SLM;
            a11 += 1.0; a12 += ex; a13 += ey;
            a22 += ex * ex; a23 += ex * ey; a33 += ey * ey;
            f0 += val; f1 += val * ex; f2 += val * ey;
        }
        if (nfin < 3) return fallback;
        double a21 = a12, a31 = a13, a32 = a23;
        double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                     a11 * a23 * a32;
        if (fabs(det) < 1e-12 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return fallback;
        double inv = 1.0 / fabs(det);
        double b11 = a22 * a33 - a23 * a32, b12 = a13 * a32 - a12 * a33, b13 = a12 * a23 - a13 * a22;
        return (b11 * f0 + b12 * f1 + b13 * f2) * inv;
    }
    return fallback;
}

/* sampling.py:432-484 _interp_mid_linear_single on a (K1, N) field */
static double mid_linear(const double* field, int64_t N, const double* zm, int K1, double z, int node) {
    if (K1 == 0) return 0.0;
    if (K1 == 1) return field[node];
    if (z <= zm[0]) return field[node];
    if (z >= zm[K1 - 1]) return field[(int64_t)(K1 - 1) * N + node];
    for (int k = 0; k < K1 - 1; ++k) {
        if (z < zm[k + 1]) {
            double dz = zm[k + 1] - zm[k];
            if (dz < 1e-12) return field[(int64_t)k * N + node];
            double a = (z - zm[k]) / dz;
            return (1.0 - a) * field[(int64_t)k * N + node] + a * field[(int64_t)(k + 1) * N + node];
        }
    }
    return field[(int64_t)(K1 - 1) * N + node];
}

typedef struct {
    const OMesh* m;
    const double* values;
    int rows;                  /* 0: a 2-D (N,) field; K1 >= 1: a (K1, N) mid-layer field */
    const double* zm;          /* (K1) mid-layer depths */
    const double *lon, *lat, *z;
    const int* nearest;
    const unsigned char* alive;
    int method;
    double* out;
} SCtx;

/* sampling.py:383-429 _loop_sample_2d and :487-541 _loop_sample_mid_3d, one particle */
static void sample_body(void* ctx, int64_t i) {
    SCtx* c = (SCtx*)ctx;
    const OMesh* m = c->m;
    if ((c->alive && !c->alive[i]) || c->nearest[i] < 0) { c->out[i] = NAN; return; }
    int nn = c->nearest[i];
    if (c->rows > 0 && !c->zm) {
        /* sampling.py:876-890: an interface field (K, N) through the W
         * interpolation of the method (vertical.py:1330-1420, time_dir +1) */
        OField f;
        memset(&f, 0, sizeof f);
        f.wa = f.wb = f.wt = c->values;
        f.n = m->N;
        int wc = c->method == S_NEAREST ? 0 : c->method == S_BARYCENTRIC ? 1 : c->method == S_LEASTSQ ? 2 : 3;
        c->out[i] = w_stage(m, &f, wc, 0.0, c->lon[i], c->lat[i], c->z[i], nn, 1.0);
        return;
    }
    int32_t buf[MAX_NEIGH];
    double vals[MAX_NEIGH];
    int cnt = neigh_ring(m, nn, buf);
    for (int k = 0; k < cnt; ++k) {
        int nd = buf[k];
        if (c->rows == 0) {
            vals[k] = c->values[nd];
        } else {
            double zp = c->z[i];
            double ze = zp < m->depth[nd] ? zp : m->depth[nd];
            vals[k] = mid_linear(c->values, m->N, c->zm, c->rows, ze, nd);
        }
    }
    c->out[i] = combine_horizontal(m, vals, buf, cnt, c->lon[i], c->lat[i], nn, c->method);
}

int orc_sample(const orc_mesh* mm, const double* values, int rows, const double* zm, int64_t P, const double* lon,
               const double* lat, const double* z, const int* nearest, const unsigned char* alive, int method,
               double* out) {
    SCtx c = {(const OMesh*)mm, values, rows, zm, lon, lat, z, nearest, alive, method, out};
    par_for(P, sample_body, &c);
    return 0;
}

/* sampling.py:620-723 _sample_sigma_3d and :545-617 _loop_sample_mid_sigma:
 * an interface field (K, N) through the sigma W interpolation of the method,
 * or a mid-layer field read in each ring node's column max(depth + eta,
 * Dmin), z clamped to it, then the method's horizontal rule.  Serial: a
 * test-size checker. */
int orc_sample_sigma(const orc_mesh* mm, const double* values, int rows, const double* eta, double Dmin, int64_t P,
                     const double* lon, const double* lat, const double* z, const int* nearest,
                     const unsigned char* alive, int method, double* out) {
    const OMesh* m = (const OMesh*)mm;
    int K = m->K;
    double zm_col[512];
    if (rows >= 512) return 1;
    for (int64_t i = 0; i < P; ++i) {
        if ((alive && !alive[i]) || nearest[i] < 0) { out[i] = NAN; continue; }
        int nn = nearest[i];
        if (rows == K) {
            OField f;
            memset(&f, 0, sizeof f);
            f.wa = f.wb = f.wt = values;
            f.etaa = f.etab = f.etat = eta;
            f.n = m->N;
            OStep s;
            memset(&s, 0, sizeof s);
            s.w_code = method == S_NEAREST ? 0 : method == S_BARYCENTRIC ? 1 : method == S_LEASTSQ ? 2 : 3;
            s.td = 1.0;
            s.dt = 1.0;
            s.Dmin = Dmin;
            out[i] = w_sig(m, &f, &s, 0, lon[i], lat[i], z[i], nn);
            continue;
        }
        int32_t buf[MAX_NEIGH];
        double vals[MAX_NEIGH];
        int cnt = neigh_ring(m, nn, buf);
        for (int k = 0; k < cnt; ++k) {
            int nd = buf[k];
            double H = m->depth[nd] + eta[nd];
            if (H < Dmin) H = Dmin;
            double ze = z[i] < H ? z[i] : H;
            for (int q = 0; q < rows; ++q) zm_col[q] = (1.0 - 0.5 * (m->sigma[q] + m->sigma[q + 1])) * H;
            vals[k] = mid_linear(values, m->N, zm_col, rows, ze, nd);
        }
        out[i] = combine_horizontal(m, vals, buf, cnt, lon[i], lat[i], nn, method);
    }
    return 0;
}
