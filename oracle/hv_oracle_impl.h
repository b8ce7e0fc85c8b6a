/*
 * hv_oracle_impl.h -- body of the CPU restatement (TEST INFRASTRUCTURE ONLY;
 * see hv_oracle.h).  Included twice by hv_oracle.c with R = double / float and
 * S = d / f.  All reference citations are paths inside BanuDarius/hyper-vlasov.
 */
#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, S)

/* IDX (include/sim_structs.hpp:38) */
#define IX(i, j, k, ny, nz) (((i) * (ny) * (nz)) + ((j) * (nz)) + (k))

/* node coordinate, world_pos_to_vector (include/tools.hpp:394-401):
 * d_max * (2 i / n - 1), evaluated as ((2 * i) / n - 1) * d_max in R. */
static inline R FN(node_pos)(R d_max, int i, int n) {
    return d_max * ((R)2.0 * (R)i / (R)n - (R)1.0);
}

/* distribute_volumetric_particles_cic (include/tools.hpp:35-96), with the
 * single-thread summation order (particle index order per node). */
void FN(orc_deposit_cic)(const orc_world *w, int protons, int neutrons, const R *x, const R *y,
                         const R *z, R *rho) {
    const R dmx = (R)w->d_max[0], dmy = (R)w->d_max[1], dmz = (R)w->d_max[2];
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    const long G = (long)nx * ny * nz;
    const int total = protons + neutrons;
    for (long i = 0; i < 2 * G; i++) rho[i] = (R)0.0;
    for (int i = 0; i < total; i++) {
        /* tools.hpp:50-52 */
        R cx = (nx / (R)2.0) * (x[i] / dmx + (R)1.0);
        R cy = (ny / (R)2.0) * (y[i] / dmy + (R)1.0);
        R cz = (nz / (R)2.0) * (z[i] / dmz + (R)1.0);
        /* tools.hpp:54-55: particles outside [0, n) on any axis are dropped */
        if (cx < (R)0.0 || cy < (R)0.0 || cz < (R)0.0 || cx >= nx || cy >= ny || cz >= nz) continue;
        int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
        int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
        R d_x = cx - x0, d_y = cy - y0, d_z = cz - z0;
        R t_x = (R)1.0 - d_x, t_y = (R)1.0 - d_y, t_z = (R)1.0 - d_z;
        long off = (i < protons) ? 0 : G;
        /* tools.hpp:64-94: corner order 000,100,010,110,001,101,011,111;
         * corners with an index equal to n are dropped */
        rho[IX(x0, y0, z0, ny, nz) + off] += t_x * t_y * t_z;
        if (x1 < nx) rho[IX(x1, y0, z0, ny, nz) + off] += d_x * t_y * t_z;
        if (y1 < ny) rho[IX(x0, y1, z0, ny, nz) + off] += t_x * d_y * t_z;
        if (x1 < nx && y1 < ny) rho[IX(x1, y1, z0, ny, nz) + off] += d_x * d_y * t_z;
        if (z1 < nz) rho[IX(x0, y0, z1, ny, nz) + off] += t_x * t_y * d_z;
        if (x1 < nx && z1 < nz) rho[IX(x1, y0, z1, ny, nz) + off] += d_x * t_y * d_z;
        if (y1 < ny && z1 < nz) rho[IX(x0, y1, z1, ny, nz) + off] += t_x * d_y * d_z;
        if (x1 < nx && y1 < ny && z1 < nz) rho[IX(x1, y1, z1, ny, nz) + off] += d_x * d_y * d_z;
    }
}

/* Offset table of the smoothing stencil: the pairs (i, j) with
 * |r_i - r_j|^2 <= 16 sigma_r^2 (include/physics.hpp:205-206,217-219), listed in
 * increasing (a, b, c) = j - i, which is the order in which the reference's
 * linear j loop meets them.  Weights exp(-d^2 / (2 sigma_r^2)) (physics.hpp:221). */
typedef struct {
    int a, b, c;
    R wgt;
} FN(orc_tap);

static int FN(build_table)(const orc_world *w, double sigma_r_d, FN(orc_tap) * taps, int cap) {
    const R sigma_r = (R)sigma_r_d;
    const R exp_term = (R)1.0 / ((R)2.0 * sigma_r * sigma_r);
    const R cutoff = (R)16.0 * sigma_r * sigma_r;
    int lim[3], ctr[3];
    R dm[3];
    for (int ax = 0; ax < 3; ax++) {
        dm[ax] = (R)w->d_max[ax];
        double h = 2.0 * w->d_max[ax] / w->n[ax];
        lim[ax] = (int)(4.0 * sigma_r_d / h) + 2;
        if (lim[ax] > w->n[ax] - 1) lim[ax] = w->n[ax] - 1;
        ctr[ax] = w->n[ax] / 2;
    }
    int count = 0;
    for (int a = -lim[0]; a <= lim[0]; a++)
        for (int b = -lim[1]; b <= lim[1]; b++)
            for (int c = -lim[2]; c <= lim[2]; c++) {
                /* r_i - r_j with i the grid centre and j = i + (a, b, c) (physics.hpp:216) */
                R d0 = FN(node_pos)(dm[0], ctr[0], w->n[0]) - FN(node_pos)(dm[0], ctr[0] + a, w->n[0]);
                R d1 = FN(node_pos)(dm[1], ctr[1], w->n[1]) - FN(node_pos)(dm[1], ctr[1] + b, w->n[1]);
                R d2 = FN(node_pos)(dm[2], ctr[2], w->n[2]) - FN(node_pos)(dm[2], ctr[2] + c, w->n[2]);
                R dist2 = d0 * d0 + d1 * d1 + d2 * d2; /* dot (math_functions.hpp:45-48) */
                if (dist2 > cutoff) continue;
                if (taps && count < cap) {
                    taps[count].a = a;
                    taps[count].b = b;
                    taps[count].c = c;
                    taps[count].wgt = EXPR(-dist2 * exp_term);
                }
                count++;
            }
    return count;
}

int FN(orc_smooth_table_size)(const orc_world *w, double sigma_r) {
    return FN(build_table)(w, sigma_r, 0, 0);
}

/* compute_volumetric_densities (include/physics.hpp:202-234). */
void FN(orc_smooth)(const orc_world *w, double sigma_r_d, int ppn, R *rho, R *tmp) {
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    const long G = (long)nx * ny * nz;
    int ntap = FN(build_table)(w, sigma_r_d, 0, 0);
    FN(orc_tap) *taps = (FN(orc_tap) *)malloc(sizeof(FN(orc_tap)) * (size_t)(ntap > 0 ? ntap : 1));
    FN(build_table)(w, sigma_r_d, taps, ntap);
    for (long i = 0; i < 2 * G; i++) tmp[i] = rho[i]; /* physics.hpp:208 */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < 2 * G; i++) {
        long node = i % G, off = (i < G) ? 0 : G;
        int ix = (int)(node / ((long)ny * nz)), iy = (int)((node / nz) % ny), iz = (int)(node % nz);
        R rho_f = (R)0.0;
        for (int t = 0; t < ntap; t++) {
            int jx = ix + taps[t].a, jy = iy + taps[t].b, jz = iz + taps[t].c;
            if (jx < 0 || jx >= nx || jy < 0 || jy >= ny || jz < 0 || jz >= nz) continue;
            R r = tmp[IX(jx, jy, jz, ny, nz) + off];
            rho_f += r * taps[t].wgt; /* physics.hpp:222 */
        }
        rho[i] = rho_f;
    }
    free(taps);
    /* physics.hpp:229-232 */
    const R sigma_r = (R)sigma_r_d;
    R term = ((R)1.0 / ppn) *
             ((R)1.0 / POWR((R)2.0 * (R)ORC_PI * sigma_r * sigma_r, (R)1.5));
    for (long i = 0; i < 2 * G; i++) rho[i] *= term;
}

/* skyrme_potential (include/physics_formulas.hpp:70-77) */
static inline R FN(skyrme_u)(R A, R B, R C, R gamma, R rho_p, R rho_n, int proton) {
    R tau = proton ? (R)-1.0 : (R)+1.0;
    R rho = rho_p + rho_n;
    R t = rho / (R)0.16;
    return A * t + B * POWR(t, gamma) + (R)2.0 * tau * C * ((rho_n - rho_p) / (R)0.16);
}

/* compute_volumetric_skyrme_potentials (include/physics.hpp:272-281) */
void FN(orc_skyrme)(const orc_world *w, const orc_skyrme *s, const R *rho, R *U) {
    const long G = (long)w->n[0] * w->n[1] * w->n[2];
    const R A = (R)s->A, B = (R)s->B, C = (R)s->C, g = (R)s->gamma;
    for (long i = 0; i < G; i++) U[i] = FN(skyrme_u)(A, B, C, g, rho[i], rho[i + G], 1);
    for (long i = G; i < 2 * G; i++) U[i] = FN(skyrme_u)(A, B, C, g, rho[i - G], rho[i], 0);
}

/* set_initial_coulomb_boundaries (include/tools.hpp:283-300) */
void FN(orc_coulomb_boundary)(const orc_world *w, int z, R *phi) {
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                if (!(i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1)) continue;
                R v0 = FN(node_pos)((R)w->d_max[0], i, nx);
                R v1 = FN(node_pos)((R)w->d_max[1], j, ny);
                R v2 = FN(node_pos)((R)w->d_max[2], k, nz);
                R r = SQRTR(v0 * v0 + v1 * v1 + v2 * v2); /* magnitude (math_functions.hpp:51-54) */
                phi[IX(i, j, k, ny, nz)] = (R)1.44 * z / r;
            }
}

/* ||b + lap_h phi||_2 / ||b||_2 over interior nodes, b = 4 pi 1.44 rho_p, in double. */
double FN(orc_rel_residual)(const orc_world *w, const R *phi, const R *rho) {
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    const double dx = 2.0 * w->d_max[0] / nx, dy = 2.0 * w->d_max[1] / ny, dz = 2.0 * w->d_max[2] / nz;
    const double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy), iz2 = 1.0 / (dz * dz);
    const double diag = 2.0 * ix2 + 2.0 * iy2 + 2.0 * iz2;
    const double c = 4.0 * ORC_PI * 1.44;
    double rr = 0.0, bb = 0.0;
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                long id = IX(i, j, k, ny, nz);
                double b = c * (double)rho[id];
                double lap = ((double)phi[IX(i + 1, j, k, ny, nz)] + (double)phi[IX(i - 1, j, k, ny, nz)]) * ix2 +
                             ((double)phi[IX(i, j + 1, k, ny, nz)] + (double)phi[IX(i, j - 1, k, ny, nz)]) * iy2 +
                             ((double)phi[IX(i, j, k + 1, ny, nz)] + (double)phi[IX(i, j, k - 1, ny, nz)]) * iz2 -
                             diag * (double)phi[id];
                double r = b + lap;
                rr += r * r;
                bb += b * b;
            }
    if (bb == 0.0) return sqrt(rr);
    return sqrt(rr / bb);
}

/* compute_volumetric_coulomb_potentials_sor (include/physics.hpp:99-157) with
 * omega, stopping rule, tolerance and cap as arguments.  Returns iterations. */
int FN(orc_sor)(const orc_world *w, R *phi, const R *rho, double omega_d, int criterion,
                double tol, int max_iter, double *metric) {
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    const R dx = (R)2.0 * (R)w->d_max[0] / nx, dy = (R)2.0 * (R)w->d_max[1] / ny,
            dz = (R)2.0 * (R)w->d_max[2] / nz;
    const R inv_dx2 = (R)1.0 / ((R)2.0 / (dx * dx) + (R)2.0 / (dy * dy) + (R)2.0 / (dz * dz));
    const R omega = (R)omega_d;
    const R src = (R)4.0 * (R)ORC_PI * (R)1.44;
    R max_diff = (R)0.0;
    double m = 0.0;
    int it;
    for (it = 0; it < max_iter; it++) {
        max_diff = (R)0.0;
        for (int color = 0; color < 2; color++) { /* red: (i+j+k) even, then black */
#pragma omp parallel for collapse(2) reduction(max : max_diff) schedule(static)
            for (int i = 1; i < nx - 1; i++)
                for (int j = 1; j < ny - 1; j++) {
                    int k0 = 1 + ((i + j + 1 + color) & 1);
                    for (int k = k0; k < nz - 1; k += 2) {
                        long id = IX(i, j, k, ny, nz);
                        R r = rho[id];
                        R phi_x = (phi[IX(i + 1, j, k, ny, nz)] + phi[IX(i - 1, j, k, ny, nz)]) / (dx * dx);
                        R phi_y = (phi[IX(i, j + 1, k, ny, nz)] + phi[IX(i, j - 1, k, ny, nz)]) / (dy * dy);
                        R phi_z = (phi[IX(i, j, k + 1, ny, nz)] + phi[IX(i, j, k - 1, ny, nz)]) / (dz * dz);
                        R phi_star = (phi_x + phi_y + phi_z + src * r) * inv_dx2;
                        R phi_old = phi[id];
                        phi[id] = ((R)1.0 - omega) * phi_old + omega * phi_star;
                        R diff = FABSR(phi[id] - phi_old);
                        if (diff > max_diff) max_diff = diff;
                    }
                }
        }
        if (criterion == 0) {
            m = (double)max_diff;
            if (max_diff < (R)tol) { it++; break; } /* physics.hpp:152-153 */
        } else {
            m = FN(orc_rel_residual)(w, phi, rho);
            if (m <= tol) { it++; break; }
        }
    }
    if (metric) *metric = m;
    return it;
}

/* merge_volumetric_potentials (include/tools.hpp:377-384) */
void FN(orc_merge)(const orc_world *w, R *U, const R *phi) {
    const long G = (long)w->n[0] * w->n[1] * w->n[2];
    for (long i = 0; i < G; i++) U[i] += phi[i];
}

/* compute_volumetric_forces_fdm (include/physics.hpp:159-200) */
void FN(orc_fdm)(const orc_world *w, const R *U, R *Fx, R *Fy, R *Fz) {
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    const long G = (long)nx * ny * nz;
    const R dx = (R)2.0 * (R)w->d_max[0] / nx, dy = (R)2.0 * (R)w->d_max[1] / ny,
            dz = (R)2.0 * (R)w->d_max[2] / nz;
    for (int s = 0; s < 2; s++) {
        const long o = s ? G : 0;
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++)
                for (int k = 0; k < nz; k++) {
                    long id = IX(i, j, k, ny, nz);
                    R gx, gy, gz;
                    if (i == 0) gx = (U[IX(1, j, k, ny, nz) + o] - U[id + o]) / dx;
                    else if (i == nx - 1) gx = (U[id + o] - U[IX(nx - 2, j, k, ny, nz) + o]) / dx;
                    else gx = (U[IX(i + 1, j, k, ny, nz) + o] - U[IX(i - 1, j, k, ny, nz) + o]) / ((R)2.0 * dx);
                    if (j == 0) gy = (U[IX(i, 1, k, ny, nz) + o] - U[id + o]) / dy;
                    else if (j == ny - 1) gy = (U[id + o] - U[IX(i, ny - 2, k, ny, nz) + o]) / dy;
                    else gy = (U[IX(i, j + 1, k, ny, nz) + o] - U[IX(i, j - 1, k, ny, nz) + o]) / ((R)2.0 * dy);
                    if (k == 0) gz = (U[IX(i, j, 1, ny, nz) + o] - U[id + o]) / dz;
                    else if (k == nz - 1) gz = (U[id + o] - U[IX(i, j, nz - 2, ny, nz) + o]) / dz;
                    else gz = (U[IX(i, j, k + 1, ny, nz) + o] - U[IX(i, j, k - 1, ny, nz) + o]) / ((R)2.0 * dz);
                    Fx[id + o] = -gx;
                    Fy[id + o] = -gy;
                    Fz[id + o] = -gz;
                }
    }
}

/* distribute_forces_to_particles_cic (include/tools.hpp:98-168) */
void FN(orc_gather_cic)(const orc_world *w, int protons, int neutrons, const R *x, const R *y,
                        const R *z, const R *Fx, const R *Fy, const R *Fz, R *fx, R *fy, R *fz) {
    const R dmx = (R)w->d_max[0], dmy = (R)w->d_max[1], dmz = (R)w->d_max[2];
    const int nx = w->n[0], ny = w->n[1], nz = w->n[2];
    const long G = (long)nx * ny * nz;
    const int total = protons + neutrons;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < total; i++) {
        R cx = (nx / (R)2.0) * (x[i] / dmx + (R)1.0);
        R cy = (ny / (R)2.0) * (y[i] / dmy + (R)1.0);
        R cz = (nz / (R)2.0) * (z[i] / dmz + (R)1.0);
        if (cx < (R)0.0 || cy < (R)0.0 || cz < (R)0.0 || cx >= nx || cy >= ny || cz >= nz) {
            fx[i] = (R)0.0; fy[i] = (R)0.0; fz[i] = (R)0.0; /* tools.hpp:112-115 */
            continue;
        }
        int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
        int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
        R d_x = cx - x0, d_y = cy - y0, d_z = cz - z0;
        R t_x = (R)1.0 - d_x, t_y = (R)1.0 - d_y, t_z = (R)1.0 - d_z;
        long off = (i < protons) ? 0 : G;
        R ax = (R)0.0, ay = (R)0.0, az = (R)0.0, wt;
        long id;
#define ORC_ACC(I, J, K, W)                     \
    id = IX(I, J, K, ny, nz) + off;             \
    wt = (W);                                   \
    ax += wt * Fx[id];                          \
    ay += wt * Fy[id];                          \
    az += wt * Fz[id];
        ORC_ACC(x0, y0, z0, t_x * t_y * t_z)
        if (x1 < nx) { ORC_ACC(x1, y0, z0, d_x * t_y * t_z) }
        if (y1 < ny) { ORC_ACC(x0, y1, z0, t_x * d_y * t_z) }
        if (x1 < nx && y1 < ny) { ORC_ACC(x1, y1, z0, d_x * d_y * t_z) }
        if (z1 < nz) { ORC_ACC(x0, y0, z1, t_x * t_y * d_z) }
        if (x1 < nx && z1 < nz) { ORC_ACC(x1, y0, z1, d_x * t_y * d_z) }
        if (y1 < ny && z1 < nz) { ORC_ACC(x0, y1, z1, t_x * d_y * d_z) }
        if (x1 < nx && y1 < ny && z1 < nz) { ORC_ACC(x1, y1, z1, d_x * d_y * d_z) }
#undef ORC_ACC
        fx[i] = ax;
        fy[i] = ay;
        fz[i] = az;
    }
}

/* update_momenta_half (include/physics.hpp:248-258) */
void FN(orc_kick_half)(int total, R *kx, R *ky, R *kz, const R *fx, const R *fy, const R *fz, R dt) {
    R fact = dt / ((R)2.0 * (R)197.33);
    for (int i = 0; i < total; i++) {
        kx[i] += fact * fx[i];
        ky[i] += fact * fy[i];
        kz[i] += fact * fz[i];
    }
}

/* update_positions_full (include/physics.hpp:260-270) */
void FN(orc_drift)(int total, R *x, R *y, R *z, const R *kx, const R *ky, const R *kz, R dt) {
    R fact = (dt * (R)197.33) / (R)935.0;
    for (int i = 0; i < total; i++) {
        x[i] += fact * kx[i];
        y[i] += fact * ky[i];
        z[i] += fact * kz[i];
    }
}

/* nuclear_excitation (include/physics.hpp:236-246) */
void FN(orc_excite)(int protons, int neutrons, R *kz, int Z, int N, R eta) {
    R zz = (R)Z, nn = (R)N;
    for (int i = 0; i < protons; i++) kz[i] += eta * nn / (zz + nn);
    for (int i = protons; i < protons + neutrons; i++) kz[i] -= eta * zz / (zz + nn);
}

/* center_of_mass (include/tools.hpp:327-338), mean_squared_radius
 * (include/tools.hpp:302-325), D (scripts/programs.py:99); sums in double. */
void FN(orc_observe)(const orc_world *w, int protons, int neutrons, const R *x, const R *y,
                     const R *z, orc_obs *out) {
    const R dmx = (R)w->d_max[0], dmy = (R)w->d_max[1], dmz = (R)w->d_max[2];
    double zs[2] = {0.0, 0.0}, r2s[2] = {0.0, 0.0};
    long cnt[2] = {0, 0};
    for (int i = 0; i < protons + neutrons; i++) {
        int s = (i < protons) ? 0 : 1;
        zs[s] += (double)z[i];
        if (x[i] < -dmx || x[i] > +dmx || y[i] < -dmy || y[i] > +dmy || z[i] < -dmz || z[i] > +dmz)
            continue;
        R r2 = x[i] * x[i] + y[i] * y[i] + z[i] * z[i];
        r2s[s] += (double)r2;
        cnt[s]++;
    }
    out->zcm_p = zs[0] / (double)protons;
    out->zcm_n = zs[1] / (double)neutrons;
    out->rms_p = sqrt(r2s[0] / (double)cnt[0]);
    out->rms_n = sqrt(r2s[1] / (double)cnt[1]);
}

/* compute_particle_densities (include/tools.hpp:170-203): for every particle
 * i, the sum over all particles j (itself included, j in index order) within
 * |r_i - r_j|^2 <= 16 sigma_r^2 of exp(-|r_i - r_j|^2 / (2 sigma_r^2)), by
 * the species of j, times 1 / (ppn (2 pi sigma_r^2)^1.5); differences r_i - r_j
 * and their dot product as sub_vec / dot (include/math_functions.hpp:42-68). */
void FN(orc_particle_densities)(int protons, int neutrons, const R *x, const R *y, const R *z,
                                double sigma_r_d, int ppn, R *dp, R *dn) {
    const int total = protons + neutrons;
    const R sigma_r = (R)sigma_r_d, exp_term = (R)1.0 / ((R)2.0 * sigma_r * sigma_r);
    const R cutoff = (R)16.0 * sigma_r * sigma_r;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < total; i++) {
        R a = (R)0.0, b = (R)0.0;
        for (int j = 0; j < total; j++) {
            const R ex = x[i] - x[j], ey = y[i] - y[j], ez = z[i] - z[j];
            const R d2 = ex * ex + ey * ey + ez * ez;
            if (d2 > cutoff) continue;
            const R f = EXPR(-d2 * exp_term);
            if (j < protons) a += f;
            else b += f;
        }
        dp[i] = a;
        dn[i] = b;
    }
    const R term = ((R)1.0 / ppn) * ((R)1.0 / POWR((R)2.0 * (R)ORC_PI * sigma_r * sigma_r, (R)1.5));
    for (int i = 0; i < total; i++) {
        dp[i] *= term;
        dn[i] *= term;
    }
}

/* cpu_simulate (src/hyper_vlasov.cpp:32-104) without VTK/stats I/O; one
 * observable row per step, recorded where the reference records it. */
int FN(orc_simulate)(const orc_world *w, const orc_run *run, int protons, int neutrons, R *x, R *y,
                     R *z, R *kx, R *ky, R *kz, int steps, orc_obs *obs, R *fields_out,
                     double *step_seconds) {
    double t0 = orc_wtime();
    const long G = (long)w->n[0] * w->n[1] * w->n[2];
    const int total = protons + neutrons;
    R *rho = (R *)calloc((size_t)(2 * G), sizeof(R));
    R *tmp = (R *)calloc((size_t)(2 * G), sizeof(R));
    R *U = (R *)calloc((size_t)(2 * G), sizeof(R));
    R *phi = (R *)calloc((size_t)G, sizeof(R));
    R *Fx = (R *)calloc((size_t)(2 * G), sizeof(R));
    R *Fy = (R *)calloc((size_t)(2 * G), sizeof(R));
    R *Fz = (R *)calloc((size_t)(2 * G), sizeof(R));
    R *fx = (R *)calloc((size_t)(total > 0 ? total : 1), sizeof(R));
    R *fy = (R *)calloc((size_t)(total > 0 ? total : 1), sizeof(R));
    R *fz = (R *)calloc((size_t)(total > 0 ? total : 1), sizeof(R));
    const R dt = (R)run->dt;
    const double nz_over_a = (double)run->n * run->z / (double)(run->n + run->z);
    int excited = 0, rc = 0;
    double metric;

    FN(orc_deposit_cic)(w, protons, neutrons, x, y, z, rho);
    FN(orc_smooth)(w, run->sigma_r, run->part_per_nucleon, rho, tmp);
    FN(orc_coulomb_boundary)(w, run->z, phi);
    FN(orc_skyrme)(w, &run->skyrme, rho, U);
    FN(orc_sor)(w, phi, rho, run->sor_omega, run->sor_criterion, run->sor_tol, run->sor_max_iter, &metric);
    FN(orc_merge)(w, U, phi);
    FN(orc_fdm)(w, U, Fx, Fy, Fz);
    FN(orc_gather_cic)(w, protons, neutrons, x, y, z, Fx, Fy, Fz, fx, fy, fz);
    if (step_seconds) step_seconds[0] = orc_wtime() - t0;
    for (int step = 0; step < steps; step++) {
        double ts = orc_wtime();
        if (obs) {
            FN(orc_observe)(w, protons, neutrons, x, y, z, &obs[step]);
            obs[step].t = (double)(step * dt);
            obs[step].dipole = nz_over_a * (obs[step].zcm_p - obs[step].zcm_n);
        }
        if (step * dt >= (R)run->t_exc && !excited) { /* hyper_vlasov.cpp:86-89 */
            excited = 1;
            FN(orc_excite)(protons, neutrons, kz, run->z, run->n, (R)run->eta_exc);
        }
        FN(orc_kick_half)(total, kx, ky, kz, fx, fy, fz, dt);
        FN(orc_drift)(total, x, y, z, kx, ky, kz, dt);
        FN(orc_deposit_cic)(w, protons, neutrons, x, y, z, rho);
        FN(orc_smooth)(w, run->sigma_r, run->part_per_nucleon, rho, tmp);
        FN(orc_skyrme)(w, &run->skyrme, rho, U);
        int its = FN(orc_sor)(w, phi, rho, run->sor_omega, run->sor_criterion, run->sor_tol,
                              run->sor_max_iter, &metric);
        if (obs) obs[step].sor_iterations = its;
        FN(orc_merge)(w, U, phi);
        FN(orc_fdm)(w, U, Fx, Fy, Fz);
        FN(orc_gather_cic)(w, protons, neutrons, x, y, z, Fx, Fy, Fz, fx, fy, fz);
        FN(orc_kick_half)(total, kx, ky, kz, fx, fy, fz, dt);
        if (step_seconds) step_seconds[1 + step] = orc_wtime() - ts;
    }
    if (fields_out) { /* layout: rho(2G) U(2G) phi(G) Fx(2G) Fy(2G) Fz(2G) */
        memcpy(fields_out, rho, sizeof(R) * 2 * G);
        memcpy(fields_out + 2 * G, U, sizeof(R) * 2 * G);
        memcpy(fields_out + 4 * G, phi, sizeof(R) * G);
        memcpy(fields_out + 5 * G, Fx, sizeof(R) * 2 * G);
        memcpy(fields_out + 7 * G, Fy, sizeof(R) * 2 * G);
        memcpy(fields_out + 9 * G, Fz, sizeof(R) * 2 * G);
    }
    free(rho); free(tmp); free(U); free(phi); free(Fx); free(Fy); free(Fz);
    free(fx); free(fy); free(fz);
    return rc;
}

/* ---- initialisation ---------------------------------------------------- */

/* compute_energy (include/tools.hpp:205-224) for every particle: Woods-Saxon
 * potential of the particle's species (physics_formulas.hpp:64-68), kinetic
 * term k^2 hbar^2 c^2 / (2 m c^2) with k = |k| (physics_formulas.hpp:34-38),
 * the uniform-sphere Coulomb potential for protons (physics_formulas.hpp:79-84)
 * and the fluctuation term 3 e_kin sigma_k^2 (physics_formulas.hpp:40-44), summed
 * in that order from 0.  ws = {V0, R12, a} of protons then neutrons. */
void FN(orc_particle_energies)(int protons, int neutrons, const R *x, const R *y, const R *z,
                               const R *kx, const R *ky, const R *kz, const double *ws,
                               double sigma_k_d, int zc_i, R *energy) {
    const R hc2 = (R)197.33 * (R)197.33, ekin = hc2 / ((R)2.0 * (R)935.0);
    const R sigma_k = (R)sigma_k_d, zc = (R)zc_i;
    const R efluc = (R)3.0 * ekin * sigma_k * sigma_k;
    const int total = protons + neutrons;
    for (int i = 0; i < total; i++) {
        const int sp = i < protons ? 0 : 1;
        const R V0 = (R)ws[3 * sp], R12 = (R)ws[3 * sp + 1], a = (R)ws[3 * sp + 2];
        const R r = SQRTR(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
        const R k = SQRTR(kx[i] * kx[i] + ky[i] * ky[i] + kz[i] * kz[i]);
        R e = (R)0.0;
        e += V0 / ((R)1.0 + EXPR((r - R12) / a));
        e += (k * k) * ekin;
        if (sp == 0) {
            if (r <= R12) e += (R)1.44 * (zc - (R)1.0) / R12 * ((R)1.5 - (R)0.5 * (r / R12) * (r / R12));
            else e += (R)1.44 * (zc - (R)1.0) / r;
        }
        e += efluc;
        energy[i] = e;
    }
}

/* Sums of the Woods-Saxon fit at x = {V0, R12, a}: out[0] = f^T f, out[1..6] =
 * J^T J (00, 01, 02, 11, 12, 22), out[7..9] = J^T f, in particle order.  The
 * residual f_i = v_skyrme_i - V0 / (1 + exp((r_i - R12) / a)) and its Jacobian
 * row are evaluated in R as woods_saxon_f / woods_saxon_df do
 * (include/fit_algorithm.hpp:49-94), the parameters first rounded to R. */
static void FN(orc_ws_sums)(int n, const R *r, const R *vs, const double *x, double *out) {
    const R V0 = (R)x[0], R12 = (R)x[1], a = (R)x[2];
    for (int q = 0; q < 10; q++) out[q] = 0.0;
    for (int i = 0; i < n; i++) {
        const R e = EXPR((r[i] - R12) / a);
        const R f = vs[i] - V0 / ((R)1.0 + e);
        const R e2 = ((R)1.0 + e) * ((R)1.0 + e);
        const double j0 = (double)(-(R)1.0 / ((R)1.0 + e));
        const double j1 = (double)(-(V0 * e) / (a * e2));
        const double j2 = (double)(-(V0 * (r[i] - R12) * e) / (a * a * e2));
        const double fd = (double)f;
        out[0] += fd * fd;
        out[1] += j0 * j0; out[2] += j0 * j1; out[3] += j0 * j2;
        out[4] += j1 * j1; out[5] += j1 * j2; out[6] += j2 * j2;
        out[7] += j0 * fd; out[8] += j1 * fd; out[9] += j2 * fd;
    }
}

/* minim_woods_saxon (include/fit_algorithm.hpp:95-137) for one species: the
 * least-squares fit of V0 / (1 + exp((r - R12) / a)) to the particles' Skyrme
 * potentials, started from ws = {V0, R12, a} and written back there.  The
 * reference calls GSL's trust-region driver (gsl_multifit_nlinear_trust, default
 * parameters, at most 100 iterations, xtol = gtol = ftol = 1e-4).  GSL is not
 * part of this restatement: the solver is Levenberg-Marquardt as published by
 * Madsen, Nielsen and Tingleff (2004, algorithm 3.16: damping mu on the scaled
 * normal equations (J^T J + mu D) h = -J^T f, gain ratio rho, mu *= max(1/3,
 * 1 - (2 rho - 1)^3) on success, mu *= nu, nu *= 2 on failure, mu_0 = 1e-3),
 * with More's scaling D = running max of diag(J^T J), and the step and
 * gradient tests of GSL's manual: |h_i| <= xtol (|x_i| + xtol) for all i;
 * max_i |g_i| max(|x_i|, 1) <= gtol max(F, 1) with F = f^T f / 2 (the
 * relative-decrease test on ftol is not applied: a fit runs until its step or
 * its gradient is small).  Returns 1 or 2 for the test that stopped it, 0 when
 * max_iter ran out, -1 when the damping grew without an accepted step, -2 for
 * fewer than 3 particles (ws unchanged).  *iters: iterations taken. */
int FN(orc_fit_woods_saxon)(int n, const R *x, const R *y, const R *z, const R *dp, const R *dn,
                            int type, const orc_skyrme *skm, double *ws, int max_iter,
                            double xtol, double gtol, int *iters) {
    *iters = 0;
    if (n < 3) return -2;
    R *r = (R *)malloc(sizeof(R) * (size_t)n), *vs = (R *)malloc(sizeof(R) * (size_t)n);
    const R A = (R)skm->A, B = (R)skm->B, C = (R)skm->C, gam = (R)skm->gamma, rho0 = (R)0.16;
    const R tau = type == 0 ? (R)-1.0 : (R)1.0;
    for (int i = 0; i < n; i++) {
        r[i] = SQRTR(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
        /* skyrme_potential (include/physics_formulas.hpp:70-77) */
        const R rho = dp[i] + dn[i], t = rho / rho0;
        vs[i] = A * t + B * POWR(t, gam) + (R)2.0 * tau * C * ((dn[i] - dp[i]) / rho0);
    }
    double p[3] = {ws[0], ws[1], ws[2]}, s[10], sn[10], D[3], h[3];
    FN(orc_ws_sums)(n, r, vs, p, s);
    for (int k = 0; k < 3; k++) D[k] = 0.0;
    double mu = 1e-3, nu = 2.0;
    int status = 0, it = 0;
    static const int dg[3] = {1, 4, 6};
    for (int k = 0; k < 3; k++) D[k] = s[dg[k]] > D[k] ? s[dg[k]] : D[k];
    for (it = 1; it <= max_iter; it++) {
        /* (J^T J + mu D) h = -J^T f by Gaussian elimination, partial pivoting */
        double M[3][4] = {{s[1] + mu * D[0], s[2], s[3], -s[7]},
                          {s[2], s[4] + mu * D[1], s[5], -s[8]},
                          {s[3], s[5], s[6] + mu * D[2], -s[9]}};
        int singular = 0;
        for (int c = 0; c < 3 && !singular; c++) {
            int pv = c;
            for (int q = c + 1; q < 3; q++)
                if (fabs(M[q][c]) > fabs(M[pv][c])) pv = q;
            if (!(fabs(M[pv][c]) > 0.0)) { singular = 1; break; }
            if (pv != c)
                for (int q = 0; q < 4; q++) { double t = M[c][q]; M[c][q] = M[pv][q]; M[pv][q] = t; }
            for (int q = c + 1; q < 3; q++) {
                const double m = M[q][c] / M[c][c];
                for (int u = c; u < 4; u++) M[q][u] -= m * M[c][u];
            }
        }
        if (singular) { status = -1; break; }
        for (int c = 2; c >= 0; c--) {
            double v = M[c][3];
            for (int u = c + 1; u < 3; u++) v -= M[c][u] * h[u];
            h[c] = v / M[c][c];
        }
        const double pn[3] = {p[0] + h[0], p[1] + h[1], p[2] + h[2]};
        FN(orc_ws_sums)(n, r, vs, pn, sn);
        const double pred = 0.5 * (mu * (D[0] * h[0] * h[0] + D[1] * h[1] * h[1] + D[2] * h[2] * h[2]) -
                                   (s[7] * h[0] + s[8] * h[1] + s[9] * h[2]));
        const double rho = pred > 0.0 ? 0.5 * (s[0] - sn[0]) / pred : -1.0;
        if (rho > 0.0 && isfinite(sn[0])) {
            for (int k = 0; k < 3; k++) p[k] = pn[k];
            for (int q = 0; q < 10; q++) s[q] = sn[q];
            for (int k = 0; k < 3; k++) D[k] = s[dg[k]] > D[k] ? s[dg[k]] : D[k];
            const double t = 2.0 * rho - 1.0, shrink = 1.0 - t * t * t;
            mu *= shrink > 1.0 / 3.0 ? shrink : 1.0 / 3.0;
            nu = 2.0;
            int xs = 1;
            for (int k = 0; k < 3; k++) xs = xs && fabs(h[k]) <= xtol * (fabs(p[k]) + xtol);
            if (xs) { status = 1; break; }
            const double F = 0.5 * s[0];
            double gm = 0.0;
            for (int k = 0; k < 3; k++) {
                const double g = fabs(s[7 + k]) * (fabs(p[k]) > 1.0 ? fabs(p[k]) : 1.0);
                gm = g > gm ? g : gm;
            }
            if (gm <= gtol * (F > 1.0 ? F : 1.0)) { status = 2; break; }
        } else {
            mu *= nu;
            nu *= 2.0;
            if (!(nu < 1e30)) { status = -1; break; }
        }
    }
    if (it > max_iter) it = max_iter;
    *iters = it;
    ws[0] = p[0]; ws[1] = p[1]; ws[2] = p[2];
    free(r); free(vs);
    return status;
}


#undef IX
#undef FN
#undef CAT
#undef CAT_
