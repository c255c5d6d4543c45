/*
 * TEST ORACLE ONLY — a plain-C restatement of the reference's CPU algorithm for the SPH-VE hydro step, in FP64 with
 * no floating-point contraction. It exists to check the CUDA path; nothing in the product links or calls it. Built by
 * oracle/Makefile into oracle/liboracle.so and loaded by tests/ (and __graft_entry__.smoke()) through ctypes.
 * Parity is pinned against the reference's own known-answer fixture (sph/test/ve.cpp + example_data.txt, committed
 * as tests/golden/) and against the reference itself compiled here (oracle/_ref).
 */
#ifndef SPH_ORACLE_H
#define SPH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    double lo[3];
    double hi[3];
    int periodic[3];
} orc_box;

#define ORC_TABLE 20000

uint64_t orc_hilbert(unsigned ix, unsigned iy, unsigned iz);
void orc_hilbert_decode(uint64_t key, unsigned* ix, unsigned* iy, unsigned* iz);
void orc_sfc_keys(size_t n, const double* x, const double* y, const double* z, const orc_box* box, uint64_t* keys);
void orc_sort_by_key(size_t n, uint64_t* keys, uint32_t* perm);
size_t orc_compute_octree(size_t n, const uint64_t* sorted_keys, unsigned bucket, uint64_t* leaves, unsigned* counts,
                          size_t cap);
double orc_kernel_tables(double sinc_index, double* wh, double* whd);
double orc_sphynx_3d_k(double n);

void orc_find_neighbors(size_t n, const double* x, const double* y, const double* z, double* h, const orc_box* box,
                        unsigned ng0, unsigned ngmax, int iterate, uint32_t* nbr, unsigned* nc);

double orc_xmass(unsigned i, double K, const orc_box* box, const uint32_t* nb, unsigned cnt, const double* x,
                 const double* y, const double* z, const double* h, const double* m, const double* wh);
void orc_ve_def_gradh(unsigned i, double K, const orc_box* box, const uint32_t* nb, unsigned cnt, const double* x,
                      const double* y, const double* z, const double* h, const double* m, const double* wh,
                      const double* whd, const double* xm, double* kx, double* gradh);
void orc_iad(unsigned i, double K, const orc_box* box, const uint32_t* nb, unsigned cnt, const double* x,
             const double* y, const double* z, const double* h, const double* wh, const double* xm, const double* kx,
             double c[6]);
void orc_divv_curlv(unsigned i, double K, const orc_box* box, const uint32_t* nb, unsigned cnt, const double* x,
                    const double* y, const double* z, const double* vx, const double* vy, const double* vz,
                    const double* h, const double* const cij[6], const double* wh, const double* kx,
                    const double* xm, double* divv, double* curlv, double dv[6]);
double orc_av_switches(unsigned i, double K, const orc_box* box, const uint32_t* nb, unsigned cnt, const double* x,
                       const double* y, const double* z, const double* vx, const double* vy, const double* vz,
                       const double* h, const double* c, const double* const cij[6], const double* wh,
                       const double* kx, const double* xm, const double* divv, double dt, double alphamin,
                       double alphamax, double decay, double alpha_i);
void orc_momentum_energy(unsigned i, int avClean, double K, const orc_box* box, const uint32_t* nb, unsigned cnt,
                         const double* x, const double* y, const double* z, const double* vx, const double* vy,
                         const double* vz, const double* h, const double* m, const double* prho, const double* c,
                         const double* const cij[6], double Atmin, double Atmax, double ramp, const double* wh,
                         const double* kx, const double* xm, const double* alpha, const double* const dv[6],
                         double out[5]);

/* whole-step simulation (particles kept in SFC order, like the reference's domain at one rank) */
typedef struct orc_sim orc_sim;
orc_sim* orc_sim_create(size_t n, const double* const* fields, const uint64_t* id, const double* box_limits,
                        int periodic, const double* params);
void orc_sim_destroy(orc_sim* s);
void orc_sim_sync(orc_sim* s);
void orc_sim_sync_perm(orc_sim* s, uint32_t* permOut);
int orc_sim_forces_active(orc_sim* s, const uint8_t* active, double avDt, double* dtCourant);
void orc_sim_set_av_clean(orc_sim* s, int on);
void orc_drift(orc_sim* s, const uint32_t* idx, size_t cnt, float dt, float dtBack, const float* dtm1,
               const uint8_t* rung);
void orc_rung_positions(orc_sim* s, const uint32_t* idx, size_t cnt, float dt, const float* dtm1, const uint8_t* rung,
                        int fold);
int orc_update_h_subset(orc_sim* s, const uint32_t* idx, size_t cnt);
int orc_sim_compute_forces(orc_sim* s);
int orc_sim_integrate(orc_sim* s);
size_t orc_sim_size(const orc_sim* s);
int orc_sim_get(const orc_sim* s, const char* name, double* out);
void orc_sim_keys(const orc_sim* s, uint64_t* out);
void orc_sim_neighbors(const orc_sim* s, uint32_t* out);
void orc_sim_scalars(const orc_sim* s, double* out);

#ifdef __cplusplus
}
#endif

#endif
