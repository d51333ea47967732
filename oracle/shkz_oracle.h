/* CPU restatement of the reference pressure projection (test infrastructure;
 * see shkz_oracle.c for the reference lines each function follows). */
#ifndef SHKZ_ORACLE_H
#define SHKZ_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif
double shkzo_get_area(const double iso[2][2]);
double shkzo_fraction(double phi0, double phi1);
void shkzo_fractions(int nx, int ny, int nz,
                     const float *solid, const unsigned char *solid_active,
                     const float *fluid, const unsigned char *fluid_active,
                     double eps_solid, double eps_fluid,
                     int second_order_fluid, int second_order_solid,
                     float *area[3], float *rho[3], float *const density[3]);
long long shkzo_label(int nx, int ny, int nz, int tile, const float *fluid,
                      float *const area[3], float *const rho[3], long long *index);
long long shkzo_assemble(int nx, int ny, int nz, double dx, double dt, const float *fluid,
                         float *const area[3], float *const rho[3],
                         float *const velocity[3], float *const solid_velocity[3],
                         const long long *index, long long n_unknowns,
                         long long *indptr, long long *indices, double *data, double *rhs);
void shkzo_spmv(long long n, const long long *indptr, const long long *indices, const double *data,
                const double *x, double *y);
void shkzo_mic0_apply(long long n, const long long *indptr, const long long *indices, const double *data,
                      double omega, double min_ratio, const double *r, double *z, double *invdiag_out);
int shkzo_pcg(long long n, const long long *indptr, const long long *indices, const double *data,
              const double *rhs, double *x, double tol, int max_iterations, int use_mic0,
              double omega, double min_ratio, double *reresid_out);
void shkzo_update_velocity(int nx, int ny, int nz, double dx, double dt, const float *pressure,
                           float *const area[3], float *const rho[3], float *const solid_velocity[3],
                           float *velocity[3], unsigned char *velocity_active[3], float *const density[3]);
int shkzo_splat(int nx, int ny, int nz, double dx, long long count, const void *particles, int stride,
                int off_p, int off_v, int off_m, int off_c, int off_bullet, int splat_bullet,
                float *velocity[3], unsigned char *velocity_active[3],
                float *mass[3], float *momentum[3], unsigned char *splat_active[3]);
#ifdef __cplusplus
}
#endif
#endif
