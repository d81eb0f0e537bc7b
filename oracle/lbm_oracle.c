/*
 * lbm_oracle.c — CPU restatement of the reference time step (see lbm_oracle.h).
 * TEST INFRASTRUCTURE: the checker for the CUDA engine, never the product.
 * Built with -ffp-contract=off (oracle/Makefile) so no FMA contraction changes
 * the reference's rounding.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stddef.h>

#define Q19 19

/* D3Q19 velocity set, weights and opposites in the reference's order
 * (LatticeModel.cpp:92-192). */
static const int C19[Q19][3] = {
    {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},   {0, 0, -1}, {1, 1, 0},
    {1, -1, 0}, {1, 0, 1},  {1, 0, -1}, {-1, 1, 0}, {-1, -1, 0}, {-1, 0, 1}, {-1, 0, -1},
    {0, 1, 1},  {0, 1, -1}, {0, -1, 1}, {0, -1, -1}, {0, 0, 0}};
static const double W19[Q19] = {
    2.0 / 36.0, 2.0 / 36.0, 2.0 / 36.0, 2.0 / 36.0, 2.0 / 36.0, 2.0 / 36.0, 1.0 / 36.0,
    1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
    1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 12.0 / 36.0};
static const int OPP19[Q19] = {1, 0, 3, 2, 5, 4, 11, 10, 13, 12, 7, 6, 9, 8, 17, 16, 15, 14, 18};

const int* orc_directions(void) { return &C19[0][0]; }
const double* orc_weights(void) { return W19; }
const int* orc_opposite(void) { return OPP19; }

void orc_init(const orc_geom* g, orc_state* s) {
    /* Node::Initialize (Node.cpp:71-78): f = w, f_new = 0; f_eq zeroed by
     * resize (Node.cpp:44-50); accumulators zeroed (Simulation.cpp:66-71). */
    const int64_t n = g->n_nodes;
    for (int64_t i = 0; i < n; ++i) {
        for (int q = 0; q < Q19; ++q) {
            s->f[i * Q19 + q] = W19[q];
            s->fnew[i * Q19 + q] = 0.0;
            s->feq[i * Q19 + q] = 0.0;
        }
        s->rho[i] = 0.0;
        s->u[3 * i] = s->u[3 * i + 1] = s->u[3 * i + 2] = 0.0;
        s->velmag[i] = 0.0;
    }
    for (int64_t k = 0; k < g->n_nearwall; ++k) {
        s->wss[k] = 0.0;
        s->acc[3 * k] = s->acc[3 * k + 1] = s->acc[3 * k + 2] = 0.0;
        s->accmag[k] = 0.0;
        s->osi[k] = 0.0;
        s->tawss[k] = 0.0;
    }
}

/* Simulation::Collision, Simulation.cpp:77-232 (D3Q19 branch). */
void orc_collide(const orc_geom* g, orc_state* s) {
    const int64_t n = g->n_nodes;
    for (int64_t i = 0; i < n; ++i) {
        const double* f = s->f + i * Q19;
        double rho = 0.0;
        for (int q = 0; q < Q19; ++q) rho += f[q];
        double* u = s->u + 3 * i;
        if (g->kind[i] == 3) {
            u[0] = 0.0;
            u[1] = 0.0;
            u[2] = 0.0;
        } else {
            u[0] = ((f[0] + f[6] + f[7] + f[8] + f[9]) - (f[1] + f[10] + f[11] + f[12] + f[13])) / rho;
            u[1] = ((f[2] + f[6] + f[10] + f[14] + f[15]) - (f[3] + f[7] + f[11] + f[16] + f[17])) / rho;
            u[2] = ((f[4] + f[8] + f[12] + f[14] + f[16]) - (f[5] + f[9] + f[13] + f[15] + f[17])) / rho;
            s->velmag[i] = sqrt(pow(u[0], 2) + pow(u[1], 2) + pow(u[2], 2));
        }
        s->rho[i] = rho;
        double* feq = s->feq + i * Q19;
        double* fn = s->fnew + i * Q19;
        for (int q = 0; q < Q19; ++q) {
            const double du = u[0] * (double)C19[q][0] + u[1] * (double)C19[q][1] + u[2] * (double)C19[q][2];
            const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
            feq[q] = W19[q] * rho * (1.0 + 3.0 * du + 4.5 * du * du - 1.5 * usq);
        }
        for (int q = 0; q < Q19; ++q) fn[q] = f[q] + (1.0 / g->tau) * (feq[q] - f[q]);
    }
}

/* Simulation::Streaming, Simulation.cpp:238-263: push f_new to the
 * neighbour unless it is missing or the value is exactly zero. */
void orc_stream(const orc_geom* g, orc_state* s) {
    const int64_t n = g->n_nodes;
    for (int64_t i = 0; i < n; ++i)
        for (int q = 0; q < Q19; ++q) {
            const int64_t j = g->nbr[i * Q19 + q];
            const double v = s->fnew[i * Q19 + q];
            if (j >= 0 && v != 0.0) s->f[j * Q19 + q] = v;
        }
}

/* ---- Zou-He inlet, Boundary::ApplyBc (Boundary.cpp:111-289) --------------
 * Each of the six face branches is a row of this table. The branches are
 * independent `if`s in the reference, applied in this order, so a normal with
 * several non-zero components runs several of them. The table keeps the
 * reference's two quirks as data: the y branches prescribe u_y = 1 instead of
 * the inlet velocity (:178, :206), and the +z branch sums the -y population
 * set for the density (:239-241). */
typedef struct {
    int comp;          /* normal component tested */
    int positive;      /* branch taken when normal[comp] > 0 (1) or < 0 (0) */
    int vel_comp;      /* velocity component that is prescribed */
    int unit_velocity; /* prescribe 1.0 instead of the inlet velocity */
    int tang[9];       /* density: populations summed once, in this order */
    int out[5];        /* density: populations counted twice */
    int denom_sign;    /* density denominator 1 + denom_sign * u[vel_comp] */
    struct { int plus[3], minus[3], vcomp; } ncorr[2]; /* transverse corrections */
    struct { int dst, src; int third; int ca, sa, cb, sb; int nidx, nsign; } set[5];
} zh_branch;

static const zh_branch ZH[6] = {
    /* +x (:115-140) */
    {0, 1, 0, 0, {2, 3, 4, 5, 14, 15, 16, 17, 18}, {0, 6, 7, 8, 9}, +1,
     {{{2, 14, 15}, {3, 16, 17}, 1}, {{4, 16, 14}, {5, 15, 17}, 2}},
     {{1, 0, 1, 0, -1, 0, 0, -1, 0},
      {10, 7, 0, 0, -1, 1, +1, 0, -1},
      {11, 6, 0, 0, -1, 1, -1, 0, +1},
      {13, 8, 0, 0, -1, 2, -1, 1, +1},
      {12, 9, 0, 0, -1, 2, +1, 1, -1}}},
    /* -x (:143-168) */
    {0, 0, 0, 0, {2, 3, 4, 5, 14, 15, 16, 17, 18}, {1, 10, 11, 12, 13}, -1,
     {{{2, 14, 15}, {3, 16, 17}, 1}, {{4, 16, 14}, {5, 15, 17}, 2}},
     {{0, 1, 1, 0, +1, 0, 0, -1, 0},
      {7, 10, 0, 0, +1, 1, -1, 0, +1},
      {6, 11, 0, 0, +1, 1, +1, 0, -1},
      {8, 13, 0, 0, +1, 2, +1, 1, -1},
      {9, 12, 0, 0, +1, 2, -1, 1, +1}}},
    /* +y (:171-195) */
    {1, 1, 1, 1, {0, 1, 4, 5, 8, 9, 12, 13, 18}, {2, 6, 10, 14, 15}, +1,
     {{{0, 8, 9}, {1, 12, 13}, 0}, {{4, 8, 12}, {5, 9, 13}, 2}},
     {{3, 2, 1, 1, -1, 1, 0, -1, 0},
      {11, 6, 0, 0, -1, 1, -1, 0, +1},
      {7, 10, 0, 1, -1, 0, +1, 0, -1},
      {17, 14, 0, 1, -1, 2, -1, 1, +1},
      {16, 15, 0, 1, -1, 2, +1, 1, -1}}},
    /* -y (:197-221) */
    {1, 0, 1, 1, {0, 1, 4, 5, 8, 9, 12, 13, 18}, {3, 7, 11, 16, 17}, -1,
     {{{0, 8, 9}, {1, 12, 13}, 0}, {{4, 8, 12}, {5, 9, 13}, 2}},
     {{2, 3, 1, 1, +1, 1, 0, -1, 0},
      {6, 11, 0, 0, +1, 1, +1, 0, -1},
      {10, 7, 0, 1, +1, 0, -1, 0, +1},
      {14, 17, 0, 1, +1, 2, +1, 1, -1},
      {15, 16, 0, 1, +1, 2, -1, 1, +1}}},
    /* +z (:225-249) */
    {2, 1, 2, 0, {0, 1, 4, 5, 8, 9, 12, 13, 18}, {3, 7, 11, 16, 17}, +1,
     {{{0, 6, 7}, {1, 10, 11}, 0}, {{2, 6, 10}, {3, 7, 11}, 1}},
     {{5, 4, 1, 2, -1, 2, 0, -1, 0},
      {9, 12, 0, 0, +1, 2, -1, 0, -1},
      {13, 8, 0, 0, -1, 2, -1, 0, +1},
      {15, 16, 0, 1, +1, 2, -1, 1, -1},
      {17, 14, 0, 1, -1, 2, -1, 1, +1}}},
    /* -z (:262-288) */
    {2, 0, 2, 0, {0, 1, 2, 3, 6, 7, 10, 11, 18}, {5, 9, 13, 15, 17}, -1,
     {{{0, 6, 7}, {1, 10, 11}, 0}, {{2, 6, 10}, {3, 7, 11}, 1}},
     {{4, 5, 1, 2, +1, 2, 0, -1, 0},
      {8, 13, 0, 0, +1, 2, +1, 0, -1},
      {12, 9, 0, 0, -1, 2, +1, 0, +1},
      {14, 17, 0, 1, +1, 2, +1, 1, -1},
      {16, 15, 0, 1, -1, 2, +1, 1, +1}}},
};

/* In the `set` rows: third=1 marks the normal population, written as
 * f[src] + sa*((1/3)*rho*u[ca]); otherwise f[src] + ((1/6)*rho)*(sa*u[ca] +
 * sb*u[cb]) + nsign*N[nidx]. Each branch prescribes a single non-zero velocity
 * component, so every two-term velocity combination is exact and its operand
 * order cannot change the rounding. */
static void zou_he_node(double* f, const double normal[3], double vel) {
    for (int b = 0; b < 6; ++b) {
        const zh_branch* z = &ZH[b];
        const double nc = normal[z->comp];
        if (!(z->positive ? nc > 0 : nc < 0)) continue;
        double u[3] = {0.0, 0.0, 0.0};
        u[z->vel_comp] = z->unit_velocity ? 1.0 : vel;
        double tsum = f[z->tang[0]];
        for (int k = 1; k < 9; ++k) tsum += f[z->tang[k]];
        double osum = f[z->out[0]];
        for (int k = 1; k < 5; ++k) osum += f[z->out[k]];
        const double denom = z->denom_sign > 0 ? 1 + u[z->vel_comp] : 1 - u[z->vel_comp];
        const double rhoN = (tsum + 2 * osum) / denom;
        double N[2];
        for (int c = 0; c < 2; ++c) {
            const double d = f[z->ncorr[c].plus[0]] + f[z->ncorr[c].plus[1]] + f[z->ncorr[c].plus[2]] -
                             f[z->ncorr[c].minus[0]] - f[z->ncorr[c].minus[1]] - f[z->ncorr[c].minus[2]];
            N[c] = (1.0 / 2) * d - (1.0 / 3) * (rhoN * u[z->ncorr[c].vcomp]);
        }
        for (int k = 0; k < 5; ++k) {
            const int dst = z->set[k].dst, src = z->set[k].src;
            if (z->set[k].third) {
                const double t = (1 / 3.0) * rhoN * u[z->set[k].ca];
                f[dst] = z->set[k].sa > 0 ? f[src] + t : f[src] - t;
            } else {
                const double va = z->set[k].sa > 0 ? u[z->set[k].ca] : -u[z->set[k].ca];
                const double vb = z->set[k].sb > 0 ? u[z->set[k].cb] : -u[z->set[k].cb];
                const double t = f[src] + (1 / 6.0) * rhoN * (va + vb);
                f[dst] = z->set[k].nsign > 0 ? t + N[z->set[k].nidx] : t - N[z->set[k].nidx];
            }
        }
    }
}

void orc_inlet(const orc_geom* g, orc_state* s, double vel) {
    for (int64_t k = 0; k < g->n_inlet; ++k) zou_he_node(s->f + g->inlet[k] * Q19, g->inlet_normal, vel);
}

/* Direction whose velocity is `d` (used for the outlet's inward neighbour). */
static int direction_of(int dx, int dy, int dz) {
    for (int q = 0; q < Q19; ++q)
        if (C19[q][0] == dx && C19[q][1] == dy && C19[q][2] == dz) return q;
    return -1;
}

/* Simulation::ApplyOutletBc, Simulation.cpp:650-741: every outlet node takes
 * all populations of its inward neighbour, one step against the first signed
 * component of the outlet normal, in list order. */
void orc_outlet(const orc_geom* g, orc_state* s) {
    for (int o = 0; o < g->n_outlets; ++o) {
        const double* nrm = g->outlet_normal + 3 * o;
        int d[3] = {0, 0, 0};
        if (nrm[0] > 0) d[0] = -1;
        else if (nrm[0] < 0) d[0] = 1;
        else if (nrm[1] > 0) d[1] = -1;
        else if (nrm[1] < 0) d[1] = 1;
        else if (nrm[2] > 0) d[2] = -1;
        else if (nrm[2] < 0) d[2] = 1;
        else continue;
        const int qin = direction_of(d[0], d[1], d[2]);
        for (int64_t k = g->outlet_off[o]; k < g->outlet_off[o + 1]; ++k) {
            const int64_t i = g->outlet_nodes[k];
            const int64_t j = g->nbr[i * Q19 + qin];
            if (j < 0) continue;
            for (int q = 0; q < Q19; ++q) s->f[i * Q19 + OPP19[q]] = s->f[j * Q19 + OPP19[q]];
        }
    }
}

/* Simulation::ApplyWallBc, Simulation.cpp:746-763: in direction order, a
 * missing neighbour in direction q copies f[q] into f[opp(q)]. */
void orc_wall(const orc_geom* g, orc_state* s) {
    for (int64_t k = 0; k < g->n_wall; ++k) {
        const int64_t i = g->wall[k];
        double* f = s->f + i * Q19;
        for (int q = 0; q < Q19; ++q)
            if (g->nbr[i * Q19 + q] < 0) f[OPP19[q]] = f[q];
    }
}

double orc_wss_constant(const orc_geom* g) {
    const double phys_den = 1060;
    const double dtdt = g->dt * g->dt;
    const double dxdx = g->spacing * g->spacing * 1e-6;
    return phys_den * dtdt / dxdx;
}

/* Simulation::ComputeWallShearStress, Simulation.cpp:767-799. */
void orc_wss(const orc_geom* g, orc_state* s) {
    const double C = orc_wss_constant(g);
    for (int64_t k = 0; k < g->n_nearwall; ++k) {
        const int64_t i = g->nearwall[k];
        const double* nrm = g->nearwall_normal + 3 * k;
        const double* f = s->f + i * Q19;
        const double* feq = s->feq + i * Q19;
        double tau[3];
        for (int a = 0; a < 3; ++a) {
            double sum_alpha = 0.0;
            for (int q = 0; q < Q19; ++q) {
                double sum_k = 0.0;
                for (int b = 0; b < 3; ++b) sum_k += (double)C19[q][b] * nrm[b] * nrm[a];
                double sum_j = 0.0;
                for (int b = 0; b < 3; ++b) sum_j += (double)C19[q][b] * nrm[b] * ((double)C19[q][a] - sum_k);
                const double fne = f[q] - feq[q];
                sum_alpha += fne * sum_j;
            }
            tau[a] = C * sum_alpha;
        }
        const double w = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
        s->wss[k] = w;
        for (int a = 0; a < 3; ++a) s->acc[3 * k + a] += tau[a];
        s->accmag[k] += w;
    }
}

/* Simulation::ComputeOSIAndTAWSS, Simulation.cpp:804-826 (period 0.9,
 * pulsatile.h:53). */
void orc_osi_tawss(const orc_geom* g, orc_state* s) {
    const double period = 0.9;
    for (int64_t k = 0; k < g->n_nearwall; ++k) {
        const double tawss = s->accmag[k] / period;
        const double* a = s->acc + 3 * k;
        const double norm = sqrt(pow(a[0], 2) + pow(a[1], 2) + pow(a[2], 2));
        s->osi[k] = 0.5 * (1.0 - (norm / s->accmag[k]));
        s->tawss[k] = tawss * g->dt;
    }
}

/* Inlet waveform: Simulation::getInletVelocity (Simulation.cpp:519-534) with
 * the three polynomial pieces of pulsatile.h:55-69. */
static double poly_piece(int piece, double x) {
    switch (piece) {
        case 1:
            return (-8.579e+08 * pow(x, 8) + 4.059e+08 * pow(x, 7) - 7.817e+07 * pow(x, 6) +
                    7.994e+06 * pow(x, 5) - 4.835e+05 * pow(x, 4) + 1.782e+04 * pow(x, 3) -
                    321.6 * pow(x, 2) + 3.215 * x + 0.1423);
        case 2:
            return (-4.32e+06 * pow(x, 8) + 7.94e+06 * pow(x, 7) - 6.298e+06 * pow(x, 6) +
                    2.82e+06 * pow(x, 5) - 7.809e+05 * pow(x, 4) + 1.37e+05 * pow(x, 3) -
                    1.484e+04 * pow(x, 2) + 901.9 * x - 22.87);
        default:
            return (-5.123 * pow(x, 4) + 14.15 * pow(x, 3) - 14.21 * pow(x, 2) + 5.865 * x - 0.5696);
    }
}

double orc_pulsatile_velocity(double t, double period) {
    const double x = fmod(t, period);
    if (x >= 0 && x < (0.1 * period)) return poly_piece(1, x);
    if (x >= (0.1 * period) && x < (0.3 * period)) return poly_piece(2, x);
    if (x >= (0.3 * period) && x < (0.9 * period)) return poly_piece(3, x);
    return 0.0;
}

int64_t orc_run(const orc_geom* g, orc_state* s, int64_t steps, int pulsatile, double cte_vel,
                double* runtime) {
    for (int64_t it = 0; it < steps; ++it) {
        orc_collide(g, s);
        orc_stream(g, s);
        const double vel = pulsatile ? orc_pulsatile_velocity(*runtime, 0.9) : cte_vel;
        orc_inlet(g, s, vel);
        orc_outlet(g, s);
        orc_wall(g, s);
        orc_wss(g, s);
        if (pulsatile) {
            orc_osi_tawss(g, s);
            *runtime += g->dt;
        }
    }
    return steps;
}

int64_t orc_pulsatile_step_count(double dt) {
    double t = 0.0;
    int64_t n = 0;
    while (t <= 2.7) {
        t += dt;
        ++n;
    }
    return n;
}
