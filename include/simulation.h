/* simulation.h — collision time step and Strang-split inhomogeneous steps.
 *
 * Entry points as upstream include/simulation.h:46-131 (src/simulation.c):
 *   CollisionStep        midpoint rule on (Cc + Cd + CB)          (:105-136)
 *   InhomStepPeriodic    1/2 transport, collision, 1/2 transport  (:307-555)
 *   InhomStepDirichlet   same, boundary cells skip the collision  (:562-830)
 *   InhomStepMaxwell     same, Maxwell reflection boundaries      (:879-1165)
 *   SimulationHomogeneous / SimulationInhomogeneous*  time loops  (:1219-1341)
 *
 * The intermediate structs keep the upstream public fields numVol, vgrid and
 * vxgridMaxw (simulation.h:63-66); the FFTW plans and host scratch states of
 * upstream are replaced by a GPU workspace handle.  The whole x-domain is
 * processed in one batched GPU launch sequence per step (upstream distributes
 * x-cells over MPI ranks, src/main_inhom.c:350-351).
 */
#ifndef SIMULATION_H
#define SIMULATION_H

#include "collision.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { struct qb_workspace *ws; } collisionInterm_t;

void CollisionInterm_Create(collisionInterm_t *interm);
void CollisionInterm_Delete(collisionInterm_t *interm);

void CollisionStep(const wignerF_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double dt, const double Bext[3], collisionInterm_t *restrict_ interm, wignerF_t *restrict_ Wnext);

typedef struct
{
	unsigned int numVol;          /* number of finite volumes (x-cells) */
	double vgrid[N_GRID];         /* velocities [0:N/2-1,-N/2:-1]*(2L)/N */
	grid_t vxgridMaxw;            /* x-velocity grid for Maxwell boundaries: 0 omitted, +L added */
	struct qb_workspace *ws;      /* GPU workspace: device states, scratch, stream */
}
inhomStepInterm_t;

void InhomStepInterm_Create(const unsigned int numVol, const double L, inhomStepInterm_t *interm);
void InhomStepInterm_Delete(inhomStepInterm_t *interm);

void InhomStepPeriodic(const wignerV_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double h, const double dt, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wnext);

void InhomStepDirichlet(const wignerV_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double h, const double dt, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wnext);

void InhomStepMaxwell(const wignerV_t *restrict_ W, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double h, const double dt, const double lambda, const wignerV_t *restrict_ WMaxwL, const wignerV_t *restrict_ WMaxwR, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wnext);

typedef struct { struct qb_workspace *ws; } simulationHomInterm_t;

void SimulationHomInterm_Create(simulationHomInterm_t *interm);
void SimulationHomInterm_Delete(simulationHomInterm_t *interm);

void SimulationHomogeneous(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double dt, const unsigned int numsteps, const double Bext[3], simulationHomInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv);

void SimulationInhomogeneousPeriodic(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double h, const double dt, const unsigned int numsteps, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv);

void SimulationInhomogeneousDirichlet(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double h, const double dt, const unsigned int numsteps, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv);

void SimulationInhomogeneousMaxwell(const wignerV_t *restrict_ W0, const quadI1_t *restrict_ quadI1, const quadI2_t *restrict_ quadI2, const quadI3_t *restrict_ quadI3, const quadI1_t *restrict_ quadI4,
	const double h, const double dt, const double lambda, const wignerV_t *restrict_ WMaxwL, const wignerV_t *restrict_ WMaxwR, const unsigned int numsteps, const double *restrict_ Bext, inhomStepInterm_t *restrict_ interm, wignerV_t *restrict_ Wevolv);

#ifdef __cplusplus
}
#endif

#endif /* SIMULATION_H */
