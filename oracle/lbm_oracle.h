/*
 * lbm_oracle — CPU restatement of the reference solver's time step, used ONLY
 * as the checker of the CUDA engine (tests, smoke check, CPU baseline timing).
 * It is not part of the product and the product never calls it.
 *
 * It restates, on flattened arrays in the reference's node order
 * (Involved_Lat_, Subdomain.cpp:598-611), the FP64 step of
 * Simulation::Iterate (Simulation.cpp:538-618): Collision (:77-232),
 * Streaming (:238-263 with Node::Stream, Node.cpp:57-61), Zou-He inlet
 * (Boundary::ApplyBc, Boundary.cpp:111-289), zero-gradient outlet
 * (:650-741), wall fix-up (:746-763), wall shear stress (:767-799),
 * OSI/TAWSS (:804-826) and the pulsatile inlet waveform (:519-534,
 * pulsatile.h:55-69). Every floating-point expression keeps the reference's
 * operand order, and the library is built without FMA contraction, so its
 * output equals the reference's bit for bit; tests/test_oracle.py pins that
 * against the reference harness dumps in tests/golden/.
 *
 * Lattice: D3Q19 with the reference's direction order (LatticeModel.cpp:92-192,
 * rest direction last).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t n_nodes;
    int32_t q;                   /* 19 */
    const int64_t* nbr;          /* [n][q]: index of node x + c_q, or -1 */
    const uint8_t* kind;         /* [n]: 0 fluid, 1 inlet, 2 outlet, 3 wall */
    int64_t n_inlet;
    const int64_t* inlet;        /* inlet node list, reference order */
    double inlet_normal[3];
    int32_t n_outlets;
    const int64_t* outlet_off;   /* [n_outlets+1] offsets into outlet_nodes */
    const int64_t* outlet_nodes; /* concatenated outlet lists, reference order */
    const double* outlet_normal; /* [n_outlets][3] */
    int64_t n_wall;
    const int64_t* wall;
    int64_t n_nearwall;
    const int64_t* nearwall;     /* near-wall (WSS) node list */
    const double* nearwall_normal; /* [n_nearwall][3] */
    double tau;                  /* relaxation time (m_relaxation) */
    double dt;                   /* time step (m_dt) */
    double spacing;              /* grid spacing in mm (Geometry::spacing) */
} orc_geom;

typedef struct {
    double* f;      /* [n][q] m_distributions */
    double* fnew;   /* [n][q] m_newDistributions */
    double* feq;    /* [n][q] m_eqdistributions */
    double* rho;    /* [n] density */
    double* u;      /* [n][3] velocity */
    double* velmag; /* [n] velMag */
    double* wss;    /* [n_nearwall] wall_shear_stress */
    double* acc;    /* [n_nearwall][3] accumulated_shear_stress */
    double* accmag; /* [n_nearwall] accumulated_shear_stress_magnitude */
    double* osi;    /* [n_nearwall] */
    double* tawss;  /* [n_nearwall] */
} orc_state;

/* Lattice tables in the reference's order. */
const int* orc_directions(void); /* [19][3] */
const double* orc_weights(void); /* [19] */
const int* orc_opposite(void);   /* [19] */

void orc_init(const orc_geom* g, orc_state* s);
void orc_collide(const orc_geom* g, orc_state* s);
void orc_stream(const orc_geom* g, orc_state* s);
void orc_inlet(const orc_geom* g, orc_state* s, double vel);
void orc_outlet(const orc_geom* g, orc_state* s);
void orc_wall(const orc_geom* g, orc_state* s);
void orc_wss(const orc_geom* g, orc_state* s);
void orc_osi_tawss(const orc_geom* g, orc_state* s);
double orc_wss_constant(const orc_geom* g);
double orc_pulsatile_velocity(double t, double period);

/* Whole steps as Simulation::Iterate runs them. pulsatile != 0 selects the
 * waveform inlet and the OSI/TAWSS update; *runtime is the waveform clock
 * (total_runtime), advanced by dt per pulsatile step. Returns steps done. */
int64_t orc_run(const orc_geom* g, orc_state* s, int64_t steps, int pulsatile, double cte_vel,
                double* runtime);

/* Number of steps Iterate performs in pulsatile mode for time step dt
 * (loop condition total_runtime <= 2.7, Simulation.cpp:549-550). */
int64_t orc_pulsatile_step_count(double dt);

#ifdef __cplusplus
}
#endif

#endif
