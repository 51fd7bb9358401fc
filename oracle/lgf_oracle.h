/*
 * CPU ORACLE — test infrastructure, not the product.
 *
 * A plain-C restatement of the LGF reference's Wilson-flow path
 * (adrian2208/msc_project, LGF/): SU(3) arithmetic, staple, flow gradient,
 * Cayley-Hamilton exponential, Luscher RK3 step, clover / improved field
 * strength, energy density E and topological charge Q.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, and
 * only as the checker.  It is pinned against the reference itself
 * (oracle/_ref/lgf_ref built from the unmodified sources, and the golden
 * vectors under tests/golden/ made from it).
 *
 * Link layout ("file order", the reference's saved-configuration layout,
 * LGF/Field/SU3_field.cpp:329-332): double L[((g*4 + mu)*9 + k)*2 + c]
 * with g the global site index ((x0*N1 + x1)*N2 + x2)*N3 + x3 (x0 slowest,
 * LGF/Lattice/Lattice.cpp:423-436), mu = 0..3, k = 3*row + col, c = re/im.
 */
#ifndef LGF_ORACLE_H
#define LGF_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

long long lgfo_volume(const int shape[4]);

/* SU3_field::staple (LGF/Field/SU3_field.cpp:519-530) */
void lgfo_staple(const double* U, const int shape[4], long long site, int mu, double out[18]);
/* Wilson::calculate_FlowGradient, one link (LGF/Action/Gauge/Wilson.cpp:55-71) */
void lgfo_flow_gradient(const double* U, const int shape[4], long long site, int mu, double out[18]);
/* HermTrLessExp: exp of an anti-Hermitian traceless iP (LGF/Math/SU3_mat.cpp:216-289) */
void lgfo_exp_iP(const double iP[18], double out[18]);
void lgfo_exp_iP_many(const double* iP, double* out, long long n);
/* GradientFlow::flow without measurement (LGF/Gradient_Flow/GradientFlow.cpp:22-54);
 * scratch holds 3 gradient fields (3*V*4*18 doubles). */
void lgfo_rk3_step(double* U, const int shape[4], double eps, double* scratch);
/* clover_avg -> F (SU3_field.cpp:533-584) and Improved_fieldStrengthTensor
 * (SU3_field.cpp:588-597); mu != nu, any order */
void lgfo_clover_F(const double* U, const int shape[4], long long site, int mu, int nu, double out[18]);
void lgfo_improved_F(const double* U, const int shape[4], long long site, int mu, int nu, double out[18]);
/* EnergyDensity::calculate (LGF/Observables/EnergyDensity.cpp:9-34): returns E.
 * per_slice (may be NULL) receives N0 values: sum over the x0 slice / V_slice. */
double lgfo_energy_density(const double* U, const int shape[4], double* per_slice);
/* TopologicalCharge::calculate (LGF/Observables/TopologicalCharge.cpp:8-29): returns Q.
 * per_slice (may be NULL) receives N0 values: the slice's share of Q (they sum to Q). */
double lgfo_topological_charge(const double* U, const int shape[4], double* per_slice);
/* per-site densities: e(x) = sum_{mu<nu} ReTr(F F), q(x) (before the 1/(4 pi^2)) */
void lgfo_site_densities(const double* U, const int shape[4], double* e_site, double* q_site);
/* The FlowSavedGaugeConfigurations measurement sequence (LGF/LGF.cpp:178-188,
 * GradientFlow.cpp:56-58, :77-84): Q and E at t=t0, then after every
 * meas_every-th of nsteps RK3 steps.  t accumulates by += eps
 * (GradientFlow.cpp:52).  Returns the number of measurements written. */
int lgfo_flow(double* U, const int shape[4], double eps, int nsteps, int meas_every, double t0,
              double* t_out, double* E_out, double* Q_out);

/* Generator G for throughput inputs: U = HermTrLessExp(i * scale * sum_a h_a T^a),
 * T^a = lambda_a / 2 (LGF/Math/SU3_gen.cpp:3-41), h_a ~ N(0,1) from a counter-based
 * hash of (seed, link, a) (Box-Muller), identical to the engine's device generator. */
void lgfo_generate_G(const int shape[4], unsigned long long seed, double scale, double* U);
/* max over links of ||U^dagger U - 1||_F and |det U - 1| */
void lgfo_unitarity(const double* U, long long nlinks, double* max_unit_err, double* max_det_err);

#ifdef __cplusplus
}
#endif
#endif
