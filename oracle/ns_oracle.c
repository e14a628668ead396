/*
 * ns_oracle.c -- CPU restatement of TubularFlowIGA's body-fitted IGA
 * Navier-Stokes hot path.  TEST INFRASTRUCTURE ONLY: the parity tests, the
 * smoke check and the bench's CPU-baseline leg call it as the checker; the
 * product library never links it.
 *
 * Every function restates one reference routine (file:line in the reference
 * project) in plain C.  Element data use the reference's layout:
 *   C[a*64+p]   dense Bezier extraction row of basis a (p = i + 4j + 16k)
 *   X[p*3+d]    Bezier control points
 *   state[a*4+f], f = (u, v, w, p)
 * Matrices are 4x4 row-major blocks in node-graph block CSR, the layout of
 * solvers/cuda/include/BlockCsr.hpp:15-100.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define TFO_OK 0
#define TFO_SINGULAR_JACOBIAN -2
#define TFO_NONPOSITIVE_JACOBIAN -3
#define TFO_BAD_INPUT -4
#define TFO_NO_MEMORY -5
#define TFO_NOT_CONVERGED -6

/* Four-point Gauss-Legendre rule on [0,1]: Quadrature.hpp:63-66. */
static const double kGaussPoint[4] = {0.06943184420297371, 0.33000947820757187,
	0.6699905217924281, 0.9305681557970262};
static const double kGaussWeight[4] = {0.3478548451374539, 0.6521451548625461,
	0.6521451548625461, 0.3478548451374539};

void tfo_gauss_rule(double* points, double* weights)
{
	/* FullCell4x4x4VolumeQuadratureProvider::BuildRule, Quadrature.hpp:193-204:
	 * qx fastest, reference weight = wx*wy*wz/8. */
	int q = 0;
	for (int qz = 0; qz < 4; ++qz)
		for (int qy = 0; qy < 4; ++qy)
			for (int qx = 0; qx < 4; ++qx, ++q) {
				points[3*q] = kGaussPoint[qx];
				points[3*q+1] = kGaussPoint[qy];
				points[3*q+2] = kGaussPoint[qz];
				weights[q] = kGaussWeight[qx]*kGaussWeight[qy]*kGaussWeight[qz]/8.0;
			}
}

/* Cubic Bernstein polynomials and derivatives: TransportElement.hpp:120-134. */
static void bernstein1(double t, double b[4], double db[4], double d2b[4])
{
	const double s = 1.0-t;
	b[0] = s*s*s; b[1] = 3.0*s*s*t; b[2] = 3.0*s*t*t; b[3] = t*t*t;
	db[0] = -3.0*s*s; db[1] = 3.0-12.0*t+9.0*t*t; db[2] = 3.0*(2.0-3.0*t)*t; db[3] = 3.0*t*t;
	d2b[0] = 6.0*s; d2b[1] = -12.0+18.0*t; d2b[2] = 6.0-18.0*t; d2b[3] = 6.0*t;
}

static void bernstein3(double u, double v, double w, double* B, double (*dB)[3], double (*d2B)[3][3])
{
	double b[3][4], db[3][4], d2b[3][4];
	bernstein1(u, b[0], db[0], d2b[0]);
	bernstein1(v, b[1], db[1], d2b[1]);
	bernstein1(w, b[2], db[2], d2b[2]);
	int p = 0;
	for (int k = 0; k < 4; ++k)
		for (int j = 0; j < 4; ++j)
			for (int i = 0; i < 4; ++i, ++p) {
				B[p] = b[0][i]*b[1][j]*b[2][k];
				dB[p][0] = db[0][i]*b[1][j]*b[2][k];
				dB[p][1] = b[0][i]*db[1][j]*b[2][k];
				dB[p][2] = b[0][i]*b[1][j]*db[2][k];
				if (d2B) {
					d2B[p][0][0] = d2b[0][i]*b[1][j]*b[2][k];
					d2B[p][0][1] = db[0][i]*db[1][j]*b[2][k];
					d2B[p][0][2] = db[0][i]*b[1][j]*db[2][k];
					d2B[p][1][0] = d2B[p][0][1];
					d2B[p][1][1] = b[0][i]*d2b[1][j]*b[2][k];
					d2B[p][1][2] = b[0][i]*db[1][j]*db[2][k];
					d2B[p][2][0] = d2B[p][0][2];
					d2B[p][2][1] = d2B[p][1][2];
					d2B[p][2][2] = b[0][i]*b[1][j]*d2b[2][k];
				}
			}
}

static double det3(const double a[3][3])
{
	/* Determinant: TransportElement.hpp:33-37. */
	return a[0][0]*a[1][1]*a[2][2]+a[0][1]*a[1][2]*a[2][0]+a[0][2]*a[1][0]*a[2][1]
		-a[0][2]*a[1][1]*a[2][0]-a[0][0]*a[1][2]*a[2][1]-a[0][1]*a[1][0]*a[2][2];
}

static int inverse3(const double a[3][3], double inv[3][3], double* determinant)
{
	/* Inverse by cofactors with the singularity guard: TransportElement.hpp:39-53. */
	const double d = det3(a);
	*determinant = d;
	if (!isfinite(d) || fabs(d) < 1e-14) return TFO_SINGULAR_JACOBIAN;
	inv[0][0] = (a[1][1]*a[2][2]-a[1][2]*a[2][1])/d;
	inv[0][1] = (a[2][1]*a[0][2]-a[0][1]*a[2][2])/d;
	inv[0][2] = (a[0][1]*a[1][2]-a[1][1]*a[0][2])/d;
	inv[1][0] = (a[2][0]*a[1][2]-a[1][0]*a[2][2])/d;
	inv[1][1] = (a[0][0]*a[2][2]-a[0][2]*a[2][0])/d;
	inv[1][2] = (a[1][0]*a[0][2]-a[0][0]*a[1][2])/d;
	inv[2][0] = (a[1][0]*a[2][1]-a[1][1]*a[2][0])/d;
	inv[2][1] = (a[0][1]*a[2][0]-a[0][0]*a[2][1])/d;
	inv[2][2] = (a[0][0]*a[1][1]-a[0][1]*a[1][0])/d;
	return TFO_OK;
}

/*
 * EvaluateBasis (TransportElement.hpp:118-206): values, physical gradients
 * and (optionally) physical Hessians of the nen extracted basis functions at
 * parametric point (u,v,w), plus J^{-1} (inverse[parameter][physical]) and
 * the raw determinant det(dx/dxi).
 */
int tfo_basis(const double* C, const double* X, int nen, double u, double v, double w,
	int with_hessian, double* N, double* dN, double* H, double* inverse_out, double* raw_det)
{
	double B[64], dB[64][3], d2B[64][3][3];
	bernstein3(u, v, w, B, dB, with_hessian ? d2B : NULL);
	double jac[3][3] = {{0}};
	for (int p = 0; p < 64; ++p)
		for (int phys = 0; phys < 3; ++phys)
			for (int par = 0; par < 3; ++par)
				jac[phys][par] += X[p*3+phys]*dB[p][par];
	double inv[3][3], det = 0.0;
	if (inverse3(jac, inv, &det) != TFO_OK) return TFO_SINGULAR_JACOBIAN;
	if (!(0.125*det > 0.0)) return TFO_NONPOSITIVE_JACOBIAN;
	double pg[64][3];
	for (int p = 0; p < 64; ++p)
		for (int phys = 0; phys < 3; ++phys) {
			double s = 0.0;
			for (int par = 0; par < 3; ++par) s += dB[p][par]*inv[par][phys];
			pg[p][phys] = s;
		}
	for (int a = 0; a < nen; ++a) {
		double value = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
		for (int p = 0; p < 64; ++p) {
			const double c = C[a*64+p];
			value += c*B[p];
			g0 += c*pg[p][0]; g1 += c*pg[p][1]; g2 += c*pg[p][2];
		}
		N[a] = value;
		dN[a*3] = g0; dN[a*3+1] = g1; dN[a*3+2] = g2;
	}
	if (inverse_out)
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < 3; ++j) inverse_out[i*3+j] = inv[i][j];
	*raw_det = det;
	if (!with_hessian) return TFO_OK;
	double gs[3][3][3] = {{{0}}};
	for (int phys = 0; phys < 3; ++phys)
		for (int p = 0; p < 64; ++p)
			for (int a = 0; a < 3; ++a)
				for (int b = 0; b < 3; ++b)
					gs[phys][a][b] += X[p*3+phys]*d2B[p][a][b];
	double is[3][3][3] = {{{0}}};
	for (int c = 0; c < 3; ++c)
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < 3; ++j)
				for (int phys = 0; phys < 3; ++phys)
					for (int a = 0; a < 3; ++a)
						for (int b = 0; b < 3; ++b)
							is[c][i][j] -= gs[phys][a][b]*inv[a][i]*inv[b][j]*inv[c][phys];
	/* Per Bernstein function, its physical Hessian; then extract. */
	double ph[64][9];
	for (int p = 0; p < 64; ++p)
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < 3; ++j) {
				double value = 0.0;
				for (int a = 0; a < 3; ++a) {
					for (int b = 0; b < 3; ++b) value += d2B[p][a][b]*inv[a][i]*inv[b][j];
					value += dB[p][a]*is[a][i][j];
				}
				ph[p][i*3+j] = value;
			}
	for (int a = 0; a < nen; ++a) {
		double h[9] = {0};
		for (int p = 0; p < 64; ++p) {
			const double c = C[a*64+p];
			if (c == 0.0) continue;
			for (int k = 0; k < 9; ++k) h[k] += c*ph[p][k];
		}
		for (int k = 0; k < 9; ++k) H[a*9+k] = h[k];
	}
	return TFO_OK;
}

/* Stabilization parameters: NavierStokesElement.hpp:121-144. */
static void stabilization(const double inv[3][3], const double state[4], double nu, double dt,
	double* tau_m, double* tau_c)
{
	double metric[3][3] = {{0}}, direction[3] = {0};
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) {
			for (int k = 0; k < 3; ++k) metric[i][j] += inv[k][i]*inv[k][j];
			direction[i] += inv[j][i];
		}
	double metric_norm = 0.0, direction_norm = 0.0, velocity_metric = 0.0;
	for (int i = 0; i < 3; ++i) {
		direction_norm += direction[i]*direction[i];
		for (int j = 0; j < 3; ++j) {
			metric_norm += metric[i][j]*metric[i][j];
			velocity_metric += state[i]*metric[i][j]*state[j];
		}
	}
	const double temporal = dt > 0.0 ? 4.0*(1.0/dt)*(1.0/dt) : 0.0;
	*tau_m = 1.0/sqrt(temporal+velocity_metric+(1.0/12.0)*nu*nu*metric_norm);
	*tau_c = 1.0/(*tau_m*direction_norm);
}

/*
 * BuildNavierStokesElementFromPreparedPoints (NavierStokesElement.hpp:149-317),
 * LegacyBodyFitted weak form, zero body force: the VMS residual (stored as
 * negres = -r) and its exact Newton tangent jac = dr/du (row 4a+i, column
 * 4b+f, dense (4 nen)^2).  jac may be NULL for the residual-only request.
 * prev may be NULL when dt == 0 (steady).
 */
int tfo_ns_element(const double* C, const double* X, int nen, const double* state,
	const double* prev, double density, double viscosity, double dt,
	const double* qpoints, const double* qweights, int nq, double* jac, double* negres)
{
	if (!(density > 0.0) || !(viscosity > 0.0) || !isfinite(dt) || dt < 0.0 || nen <= 0 || nen > 80)
		return TFO_BAD_INPUT;
	const double nu = viscosity/density;
	const int ndof = 4*nen;
	if (jac) memset(jac, 0, sizeof(double)*(size_t)ndof*ndof);
	memset(negres, 0, sizeof(double)*(size_t)ndof);
	double N[80], dN[80*3], H[80*9];
	for (int q = 0; q < nq; ++q) {
		double inv_flat[9], raw = 0.0;
		const int status = tfo_basis(C, X, nen, qpoints[3*q], qpoints[3*q+1], qpoints[3*q+2], 1,
			N, dN, H, inv_flat, &raw);
		if (status != TFO_OK) return status;
		double inv[3][3];
		for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) inv[i][j] = inv_flat[i*3+j];
		const double measure = qweights[q]*raw;
		double st[4] = {0}, grad[4][3] = {{0}}, hess[4][3][3] = {{{0}}}, pv[3] = {0};
		for (int a = 0; a < nen; ++a)
			for (int f = 0; f < 4; ++f) {
				const double c = state[a*4+f];
				st[f] += c*N[a];
				for (int i = 0; i < 3; ++i) {
					grad[f][i] += c*dN[a*3+i];
					for (int j = 0; j < 3; ++j) hess[f][i][j] += c*H[a*9+i*3+j];
				}
			}
		if (dt > 0.0)
			for (int a = 0; a < nen; ++a)
				for (int c = 0; c < 3; ++c) pv[c] += prev[a*4+c]*N[a];
		double dudt[3] = {0};
		if (dt > 0.0) for (int c = 0; c < 3; ++c) dudt[c] = (st[c]-pv[c])/dt;
		double tau_m = 0.0, tau_c = 0.0;
		stabilization(inv, st, nu, dt, &tau_m, &tau_c);
		double fine[3];
		for (int c = 0; c < 3; ++c) {
			const double conv = st[0]*grad[c][0]+st[1]*grad[c][1]+st[2]*grad[c][2];
			const double lap = hess[c][0][0]+hess[c][1][1]+hess[c][2][2];
			fine[c] = -tau_m*(dudt[c]+conv+grad[3][c]/density-nu*lap);
		}
		const double divu = grad[0][0]+grad[1][1]+grad[2][2];
		const double fine_p = -density*tau_c*divu;
		double metric[3][3] = {{0}};
		if (jac)
			for (int i = 0; i < 3; ++i)
				for (int j = 0; j < 3; ++j)
					for (int k = 0; k < 3; ++k) metric[i][j] += inv[k][i]*inv[k][j];
		/* Strong momentum residual (without tau), reused by the tangent. */
		double strong[3];
		for (int c = 0; c < 3; ++c)
			strong[c] = dudt[c]+st[0]*grad[c][0]+st[1]*grad[c][1]+st[2]*grad[c][2]
				+grad[3][c]/density-nu*(hess[c][0][0]+hess[c][1][1]+hess[c][2][2]);
		for (int a = 0; a < nen; ++a) {
			const double na = N[a];
			const double* ga = dN+a*3;
			double r[4];
			for (int c = 0; c < 3; ++c) {
				r[c] = density*na*dudt[c]-ga[c]*fine_p;
				r[c] -= ga[c]*st[3];
				for (int d = 0; d < 3; ++d) {
					r[c] += viscosity*ga[d]*(grad[c][d]+grad[d][c]);
					r[c] += density*na*(st[d]+fine[d])*grad[c][d];
					r[c] -= density*ga[d]*fine[c]*(st[d]+fine[d]);
				}
			}
			r[3] = na*divu-ga[0]*fine[0]-ga[1]*fine[1]-ga[2]*fine[2];
			for (int f = 0; f < 4; ++f) negres[4*a+f] -= r[f]*measure;
			if (!jac) continue;
			for (int b = 0; b < nen; ++b) {
				const double nb = N[b];
				const double* gb = dN+b*3;
				const double lap_b = H[b*9]+H[b*9+4]+H[b*9+8];
				for (int f = 0; f < 4; ++f) {
					double du[3] = {0}, dlap[3] = {0}, dgp[3] = {0};
					const double dp = f == 3 ? nb : 0.0;
					if (f < 3) { du[f] = nb; dlap[f] = lap_b; }
					else { dgp[0] = gb[0]; dgp[1] = gb[1]; dgp[2] = gb[2]; }
					double vmd = 0.0;
					for (int i = 0; i < 3; ++i)
						for (int j = 0; j < 3; ++j) vmd += du[i]*metric[i][j]*st[j];
					const double dtau_m = -tau_m*tau_m*tau_m*vmd;
					const double dtau_c = tau_c*tau_m*tau_m*vmd;
					const double ddiv = f < 3 ? gb[f] : 0.0;
					double dfine[3];
					for (int c = 0; c < 3; ++c) {
						double ds = 0.0;
						for (int d = 0; d < 3; ++d)
							ds += du[d]*grad[c][d]+st[d]*(f == c ? gb[d] : 0.0);
						if (dt > 0.0 && f == c) ds += nb/dt;
						ds += dgp[c]/density-nu*dlap[c];
						dfine[c] = -dtau_m*strong[c]-tau_m*ds;
					}
					const double dfine_p = -density*(dtau_c*divu+tau_c*ddiv);
					for (int i = 0; i < 3; ++i) {
						double t = density*na*(dt > 0.0 && f == i ? nb/dt : 0.0)-ga[i]*dfine_p;
						t -= ga[i]*dp;
						for (int d = 0; d < 3; ++d) {
							t += viscosity*ga[d]*((f == i ? gb[d] : 0.0)+(f == d ? gb[i] : 0.0));
							t += density*na*((du[d]+dfine[d])*grad[i][d]
								+(st[d]+fine[d])*(f == i ? gb[d] : 0.0));
							t -= density*ga[d]*(dfine[i]*(st[d]+fine[d])+fine[i]*(du[d]+dfine[d]));
						}
						jac[(size_t)(4*a+i)*ndof+4*b+f] += t*measure;
					}
					double ct = na*ddiv;
					for (int d = 0; d < 3; ++d) ct -= ga[d]*dfine[d];
					jac[(size_t)(4*a+3)*ndof+4*b+f] += ct*measure;
				}
			}
		}
	}
	return TFO_OK;
}

/* 0.125 det(dx/dxi) at the 4x4x4 Gauss points (InspectGeometry,
 * TransportElement.hpp:55-90): returns the minimum and counts bad samples. */
double tfo_min_determinant(const double* X, int* bad_samples)
{
	double minimum = INFINITY;
	int bad = 0;
	for (int k = 0; k < 4; ++k)
		for (int j = 0; j < 4; ++j)
			for (int i = 0; i < 4; ++i) {
				double B[64], dB[64][3];
				bernstein3(kGaussPoint[i], kGaussPoint[j], kGaussPoint[k], B, dB, NULL);
				double jac[3][3] = {{0}};
				for (int p = 0; p < 64; ++p)
					for (int phys = 0; phys < 3; ++phys)
						for (int par = 0; par < 3; ++par) jac[phys][par] += X[p*3+phys]*dB[p][par];
				const double d = 0.125*det3(jac);
				if (d < minimum) minimum = d;
				if (!isfinite(d) || d <= 0.0) ++bad;
			}
	if (bad_samples) *bad_samples = bad;
	return minimum;
}

/* Face tables of the body-fitted surface rule: BoundaryFlow.hpp:175-180. */
static const int kFixedAxis[6] = {2, 1, 0, 1, 0, 2};
static const int kVaryingAxes[6][2] = {{0, 1}, {0, 2}, {1, 2}, {0, 2}, {1, 2}, {0, 1}};
static const double kFixedValue[6] = {0.0, 0.0, 1.0, 1.0, 0.0, 1.0};
static const double kOutwardSign[6] = {-1.0, -1.0, 1.0, 1.0, -1.0, 1.0};

/*
 * Per-face flow coefficients F[a*3+c] such that the outward boundary flow of
 * face `face` is sum_a sum_c F[a*3+c] u_a[c] (IntegrateBoundaryFlow,
 * BoundaryFlow.hpp:165-200) and the pressure traction of pressure p adds
 * -p F[a*3+c] to rhs (IntegrateBoundaryPressureTraction, :445-475).
 */
int tfo_face_coefficients(const double* C, const double* X, int nen, int face, double* F)
{
	if (face < 0 || face >= 6) return TFO_BAD_INPUT;
	memset(F, 0, sizeof(double)*(size_t)nen*3);
	double N[80], dN[240];
	for (int qi = 0; qi < 4; ++qi)
		for (int qj = 0; qj < 4; ++qj) {
			double coordinate[3] = {0, 0, 0};
			coordinate[kFixedAxis[face]] = kFixedValue[face];
			coordinate[kVaryingAxes[face][0]] = kGaussPoint[qi];
			coordinate[kVaryingAxes[face][1]] = kGaussPoint[qj];
			double inv[9], raw = 0.0;
			const int status = tfo_basis(C, X, nen, coordinate[0], coordinate[1], coordinate[2], 0,
				N, dN, NULL, inv, &raw);
			if (status != TFO_OK) return status;
			const double scale = kOutwardSign[face]*kGaussWeight[qi]*kGaussWeight[qj]*2.0*(0.125*raw);
			for (int a = 0; a < nen; ++a)
				for (int c = 0; c < 3; ++c)
					F[a*3+c] += scale*inv[kFixedAxis[face]*3+c]*N[a];
		}
	return TFO_OK;
}

double tfo_boundary_flow(const double* C, const double* X, int nen, int face, const double* state)
{
	double F[240];
	if (tfo_face_coefficients(C, X, nen, face, F) != TFO_OK) return NAN;
	double flow = 0.0;
	for (int a = 0; a < nen; ++a)
		for (int c = 0; c < 3; ++c) flow += F[a*3+c]*state[a*4+c];
	return flow;
}

/* Outlet 0D models (EvaluateOutletModel, OutletModel.hpp:70-90).
 * kind: 0 resistance, 1 windkessel RC, 2 windkessel RCR. */
int tfo_outlet_model(int kind, double resistance, double proximal, double distal, double capacitance,
	double reference_pressure, double capacitor_pressure, double flow, double dt,
	double* pressure, double* new_capacitor_pressure)
{
	if (!isfinite(flow)) return TFO_BAD_INPUT;
	if (kind == 0) {
		*pressure = reference_pressure+resistance*flow;
		*new_capacitor_pressure = capacitor_pressure;
		return TFO_OK;
	}
	if (!(dt > 0.0)) return TFO_BAD_INPUT;
	const double r = kind == 1 ? resistance : distal;
	const double pc = (capacitance*capacitor_pressure/dt+flow+reference_pressure/r)/(capacitance/dt+1.0/r);
	*new_capacitor_pressure = pc;
	*pressure = pc+(kind == 2 ? proximal*flow : 0.0);
	return TFO_OK;
}

/* Temporal waveforms (EvaluateTemporalFunction, TemporalFunction.hpp:97-112).
 * kind: 0 constant, 1 sinusoid, 2 fourier. */
double tfo_temporal(int kind, double value, double mean, double amplitude, double period, double phase,
	const double* cosine, const double* sine, int harmonics, double time)
{
	const double pi = 3.141592653589793238462643383279502884;
	if (kind == 0) return value;
	double wrapped = fmod(time, period);
	if (wrapped < 0.0) wrapped += period;
	const double theta = 2.0*pi*wrapped/period+phase;
	if (kind == 1) return mean+amplitude*sin(theta);
	double result = mean;
	for (int h = 0; h < harmonics; ++h) {
		const double angle = (double)(h+1)*theta;
		result += cosine[h]*cos(angle)+sine[h]*sin(angle);
	}
	return result;
}

/* ---------------------------------------------------------------------- */
/* Global (mesh-level) restatements.                                      */
/* ---------------------------------------------------------------------- */

static int compare_int(const void* a, const void* b)
{
	const int x = *(const int*)a, y = *(const int*)b;
	return (x > y)-(x < y);
}

/*
 * Node-graph block pattern (BlockPattern, BlockCsr.hpp:15-55): sorted unique
 * columns per node row.  Call with columns == NULL to get the block count in
 * *blocks; then call again with arrays of that size.
 */
int tfo_block_pattern(int nodes, int elements, const int* element_offsets, const int* connectivity,
	int* row_offsets, int* columns, int* diagonal, long long* blocks)
{
	int* count = (int*)calloc((size_t)nodes+1, sizeof(int));
	if (!count) return TFO_NO_MEMORY;
	for (int e = 0; e < elements; ++e) {
		const int nen = element_offsets[e+1]-element_offsets[e];
		for (int a = element_offsets[e]; a < element_offsets[e+1]; ++a) {
			const int node = connectivity[a];
			if (node < 0 || node >= nodes) { free(count); return TFO_BAD_INPUT; }
			count[node] += nen;
		}
	}
	long long* start = (long long*)malloc(sizeof(long long)*((size_t)nodes+1));
	start[0] = 0;
	for (int i = 0; i < nodes; ++i) start[i+1] = start[i]+count[i];
	int* raw = (int*)malloc(sizeof(int)*(size_t)(start[nodes] > 0 ? start[nodes] : 1));
	memset(count, 0, sizeof(int)*((size_t)nodes+1));
	for (int e = 0; e < elements; ++e)
		for (int a = element_offsets[e]; a < element_offsets[e+1]; ++a) {
			const int node = connectivity[a];
			for (int b = element_offsets[e]; b < element_offsets[e+1]; ++b)
				raw[start[node]+count[node]++] = connectivity[b];
		}
	long long total = 0;
	for (int i = 0; i < nodes; ++i) {
		int* row = raw+start[i];
		const int length = count[i];
		qsort(row, (size_t)length, sizeof(int), compare_int);
		int unique = 0;
		for (int k = 0; k < length; ++k)
			if (unique == 0 || row[unique-1] != row[k]) row[unique++] = row[k];
		int has_diagonal = 0;
		if (columns) {
			row_offsets[i] = (int)total;
			for (int k = 0; k < unique; ++k) {
				if (row[k] == i) { diagonal[i] = (int)(total+k); has_diagonal = 1; }
				columns[total+k] = row[k];
			}
			if (!has_diagonal) { free(raw); free(start); free(count); return TFO_BAD_INPUT; }
		}
		total += unique;
	}
	if (columns) row_offsets[nodes] = (int)total;
	*blocks = total;
	free(raw); free(start); free(count);
	return TFO_OK;
}

static long long find_block(const int* row_offsets, const int* columns, int row, int column)
{
	/* FindBlock: SparseKernels.cuh:13-23. */
	int first = row_offsets[row], last = row_offsets[row+1];
	while (first < last) {
		const int middle = first+(last-first)/2;
		if (columns[middle] < column) first = middle+1;
		else last = middle;
	}
	return first;
}

/*
 * Global assembly: every element's exact tangent and -r scatter-added into
 * the block-CSR Jacobian and rhs (AddElementMatrix semantics,
 * OwnedRowAssembler.hpp:210-236; the loop of iga_cuda.cu:959-965).  The
 * element extraction is passed in the flattened sparse layout of FlatMesh
 * (DeviceMesh.hpp:16-57).  values may be NULL for a residual-only pass.
 * Element failures are reported through *failed_element (-1 = none).
 */
int tfo_assemble(int nodes, int elements, const int* element_offsets, const int* connectivity,
	const int* extraction_offsets, const uint8_t* extraction_columns, const double* extraction_values,
	const double* bezier_points, const int* row_offsets, const int* columns,
	const double* state, const double* previous, double density, double viscosity, double dt,
	double* values, double* rhs, int* failed_element)
{
	(void)nodes;
	double qp[64*3], qw[64];
	tfo_gauss_rule(qp, qw);
	int failure = -1, status_out = TFO_OK;
#pragma omp parallel
	{
		double* C = (double*)malloc(sizeof(double)*80*64);
		double* jac = values ? (double*)malloc(sizeof(double)*320*320) : NULL;
		double negres[320], st[320], pv[320];
		long long blocks[80];
#pragma omp for schedule(dynamic, 4)
		for (int e = 0; e < elements; ++e) {
			const int begin = element_offsets[e];
			const int nen = element_offsets[e+1]-begin;
			memset(C, 0, sizeof(double)*(size_t)nen*64);
			for (int a = 0; a < nen; ++a)
				for (int k = extraction_offsets[begin+a]; k < extraction_offsets[begin+a+1]; ++k)
					C[a*64+extraction_columns[k]] = extraction_values[k];
			for (int a = 0; a < nen; ++a) {
				const int node = connectivity[begin+a];
				for (int f = 0; f < 4; ++f) {
					st[4*a+f] = state[4*(size_t)node+f];
					pv[4*a+f] = previous ? previous[4*(size_t)node+f] : 0.0;
				}
			}
			const int status = tfo_ns_element(C, bezier_points+(size_t)e*192, nen, st, pv,
				density, viscosity, dt, qp, qw, 64, jac, negres);
			if (status != TFO_OK) {
#pragma omp critical
				{ failure = e; status_out = status; }
				continue;
			}
			for (int a = 0; a < nen; ++a) {
				const int row = connectivity[begin+a];
				for (int f = 0; f < 4; ++f) {
#pragma omp atomic
					rhs[4*(size_t)row+f] += negres[4*a+f];
				}
			}
			if (!values) continue;
			const int ndof = 4*nen;
			for (int a = 0; a < nen; ++a) {
				const int row = connectivity[begin+a];
				for (int b = 0; b < nen; ++b)
					blocks[b] = find_block(row_offsets, columns, row, connectivity[begin+b]);
				for (int b = 0; b < nen; ++b) {
					double* block = values+blocks[b]*16;
					for (int i = 0; i < 4; ++i)
						for (int f = 0; f < 4; ++f) {
#pragma omp atomic
							block[i*4+f] += jac[(size_t)(4*a+i)*ndof+4*b+f];
						}
				}
			}
		}
		free(C);
		free(jac);
	}
	if (failed_element) *failed_element = failure;
	return status_out;
}

/*
 * Dirichlet rows (ApplyNavierStokesBoundaryKernel / SetNavierStokesBoundaryRhsKernel,
 * IgaCudaKernels.cuh:436-463): zero the constrained rows, put 1 on the
 * diagonal, rhs = target - state.
 */
void tfo_apply_dirichlet(int nodes, const int* row_offsets, const int* diagonal,
	const int* velocity_mask, const int* pressure_mask, const double* velocity, const double* pressure,
	const double* state, double* values, double* rhs)
{
	for (int node = 0; node < nodes; ++node)
		for (int f = 0; f < 4; ++f) {
			const int constrained = f < 3 ? velocity_mask[node] : pressure_mask[node];
			if (!constrained) continue;
			if (values) {
				for (int b = row_offsets[node]; b < row_offsets[node+1]; ++b)
					for (int g = 0; g < 4; ++g) values[(size_t)b*16+f*4+g] = 0.0;
				values[(size_t)diagonal[node]*16+f*4+f] = 1.0;
			}
			const double target = f < 3 ? velocity[3*(size_t)node+f] : pressure[node];
			rhs[4*(size_t)node+f] = target-state[4*(size_t)node+f];
		}
}

/* y = A x over F x F blocks (BlockSpmvKernel<F>, SparseKernels.cuh:25-40), F <= 4. */
static void spmv_f(int F, int nodes, const int* row_offsets, const int* columns, const double* values,
	const double* x, double* y)
{
#pragma omp parallel for schedule(static)
	for (int row = 0; row < nodes; ++row) {
		double r[4] = {0, 0, 0, 0};
		for (int b = row_offsets[row]; b < row_offsets[row+1]; ++b) {
			const double* blk = values+(size_t)b*F*F;
			const double* xc = x+(size_t)F*columns[b];
			for (int i = 0; i < F; ++i)
				for (int j = 0; j < F; ++j) r[i] += blk[i*F+j]*xc[j];
		}
		for (int i = 0; i < F; ++i) y[(size_t)F*row+i] = r[i];
	}
}

void tfo_spmv(int nodes, const int* row_offsets, const int* columns, const double* values,
	const double* x, double* y)
{
	spmv_f(4, nodes, row_offsets, columns, values, x, y);
}

/* Diagonal-block Gauss-Jordan inverse with partial pivoting and the
 * singular fallback (BuildBlockInverseKernel<F>, SparseKernels.cuh:42-89), F <= 4. */
static int block_inverse_f(int F, int nodes, const int* diagonal, const double* values, double* inverse)
{
	int singular = 0;
#pragma omp parallel for schedule(static) reduction(+:singular)
	for (int node = 0; node < nodes; ++node) {
		const double* s = values+(size_t)diagonal[node]*F*F;
		double m[4][8];
		for (int i = 0; i < F; ++i)
			for (int j = 0; j < 2*F; ++j) m[i][j] = j < F ? s[i*F+j] : (j-F == i ? 1.0 : 0.0);
		int failed = 0;
		for (int pivot = 0; pivot < F; ++pivot) {
			int best = pivot;
			for (int row = pivot+1; row < F; ++row)
				if (fabs(m[row][pivot]) > fabs(m[best][pivot])) best = row;
			if (!isfinite(m[best][pivot]) || fabs(m[best][pivot]) < 1e-14) { failed = 1; break; }
			if (best != pivot)
				for (int c = 0; c < 2*F; ++c) { const double t = m[pivot][c]; m[pivot][c] = m[best][c]; m[best][c] = t; }
			const double scale = 1.0/m[pivot][pivot];
			for (int c = 0; c < 2*F; ++c) m[pivot][c] *= scale;
			for (int row = 0; row < F; ++row) {
				if (row == pivot) continue;
				const double factor = m[row][pivot];
				for (int c = 0; c < 2*F; ++c) m[row][c] -= factor*m[pivot][c];
			}
		}
		double* d = inverse+(size_t)node*F*F;
		if (!failed) {
			for (int i = 0; i < F; ++i) for (int j = 0; j < F; ++j) d[i*F+j] = m[i][F+j];
		} else {
			++singular;
			for (int i = 0; i < F; ++i)
				for (int j = 0; j < F; ++j)
					d[i*F+j] = i == j && fabs(s[i*F+i]) > 1e-14 ? 1.0/s[i*F+i] : (i == j ? 1.0 : 0.0);
		}
	}
	return singular;
}

int tfo_block_inverse(int nodes, const int* diagonal, const double* values, double* inverse)
{
	return block_inverse_f(4, nodes, diagonal, values, inverse);
}

static void apply_block_inverse_f(int F, int nodes, const double* inverse, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
	for (int node = 0; node < nodes; ++node)
		for (int i = 0; i < F; ++i) {
			double r = 0.0;
			for (int j = 0; j < F; ++j) r += inverse[((size_t)node*F+i)*F+j]*x[(size_t)F*node+j];
			y[(size_t)F*node+i] = r;
		}
}

static double dot(long long n, const double* x, const double* y)
{
	double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+:s)
	for (long long i = 0; i < n; ++i) s += x[i]*y[i];
	return s;
}

static void axpy(long long n, double alpha, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
	for (long long i = 0; i < n; ++i) y[i] += alpha*x[i];
}

/*
 * Restarted left-preconditioned GMRES(m) with modified Gram-Schmidt,
 * Givens rotations and the true-residual restart check, block-Jacobi
 * preconditioned (SolveGmres, Gmres.hpp:192-336, zero polynomial sweeps).
 * Tolerance: max(1e-30, rtol * ||D^{-1} (b - A x0)||).  Returns the
 * iteration count (>= 0) or TFO_NOT_CONVERGED; *residual gets the final
 * preconditioned residual norm.
 */
typedef void (*precond_fn)(const void* context, const double* in, double* out);

/* apply (may be NULL): the left preconditioner M^{-1}; NULL = the block-Jacobi inverse. */
static int gmres_precond_f(int F, int nodes, const int* row_offsets, const int* columns, const int* diagonal,
	const double* values, const double* rhs, double* x, int restart, int maximum_iterations,
	double rtol, double* residual_out, int* singular_out, precond_fn apply, const void* context)
{
	const long long n = (long long)F*nodes;
	double* inverse = (double*)malloc(sizeof(double)*(size_t)n*F);
	double* raw = (double*)malloc(sizeof(double)*(size_t)n);
	double* res = (double*)malloc(sizeof(double)*(size_t)n);
	double* work = (double*)malloc(sizeof(double)*(size_t)n);
	double* V = (double*)malloc(sizeof(double)*(size_t)n*(size_t)(restart+1));
	double* h = (double*)calloc((size_t)(restart+1)*restart, sizeof(double));
	double* cs = (double*)calloc((size_t)restart, sizeof(double));
	double* sn = (double*)calloc((size_t)restart, sizeof(double));
	double* g = (double*)calloc((size_t)restart+1, sizeof(double));
	double* y = (double*)calloc((size_t)restart, sizeof(double));
	if (!inverse || !raw || !res || !work || !V || !h || !cs || !sn || !g || !y) return TFO_NO_MEMORY;
	const int singular = apply ? 0 : block_inverse_f(F, nodes, diagonal, values, inverse);
	if (singular_out) *singular_out = singular;
	spmv_f(F, nodes, row_offsets, columns, values, x, raw);
	for (long long i = 0; i < n; ++i) res[i] = rhs[i]-raw[i];
	if (apply) apply(context, res, work);
	else apply_block_inverse_f(F, nodes, inverse, res, work);
	const double initial = sqrt(dot(n, work, work));
	int iterations = 0, converged = 0;
	double residual = initial;
	if (initial == 0.0) converged = 1;
	const double tolerance = fmax(1e-30, rtol*initial);
	double beta = initial;
	while (!converged && iterations < maximum_iterations) {
		for (long long i = 0; i < n; ++i) V[i] = work[i]/beta;
		memset(h, 0, sizeof(double)*(size_t)(restart+1)*restart);
		memset(g, 0, sizeof(double)*((size_t)restart+1));
		g[0] = beta;
		int used = 0;
		for (int j = 0; j < restart && iterations < maximum_iterations; ++j) {
			spmv_f(F, nodes, row_offsets, columns, values, V+(size_t)j*n, raw);
			if (apply) apply(context, raw, work);
			else apply_block_inverse_f(F, nodes, inverse, raw, work);
			for (int i = 0; i <= j; ++i) {
				const double value = dot(n, V+(size_t)i*n, work);
				h[(size_t)i*restart+j] = value;
				axpy(n, -value, V+(size_t)i*n, work);
			}
			const double next = sqrt(dot(n, work, work));
			h[(size_t)(j+1)*restart+j] = next;
			if (next > 1e-30)
				for (long long i = 0; i < n; ++i) V[(size_t)(j+1)*n+i] = work[i]/next;
			for (int i = 0; i < j; ++i) {
				const double a = h[(size_t)i*restart+j], b = h[(size_t)(i+1)*restart+j];
				h[(size_t)i*restart+j] = cs[i]*a+sn[i]*b;
				h[(size_t)(i+1)*restart+j] = -sn[i]*a+cs[i]*b;
			}
			const double a = h[(size_t)j*restart+j], b = h[(size_t)(j+1)*restart+j];
			const double mag = hypot(a, b);
			cs[j] = mag > 0.0 ? a/mag : 1.0;
			sn[j] = mag > 0.0 ? b/mag : 0.0;
			h[(size_t)j*restart+j] = mag;
			h[(size_t)(j+1)*restart+j] = 0.0;
			const double old = g[j];
			g[j] = cs[j]*old;
			g[j+1] = -sn[j]*old;
			++iterations;
			used = j+1;
			residual = fabs(g[j+1]);
			if (residual <= tolerance || next <= 1e-30) break;
		}
		for (int row = used-1; row >= 0; --row) {
			double value = g[row];
			for (int c = row+1; c < used; ++c) value -= h[(size_t)row*restart+c]*y[c];
			y[row] = value/h[(size_t)row*restart+row];
		}
		for (int i = 0; i < used; ++i) axpy(n, y[i], V+(size_t)i*n, x);
		spmv_f(F, nodes, row_offsets, columns, values, x, raw);
		for (long long i = 0; i < n; ++i) res[i] = rhs[i]-raw[i];
		if (apply) apply(context, res, work);
		else apply_block_inverse_f(F, nodes, inverse, res, work);
		beta = sqrt(dot(n, work, work));
		residual = beta;
		if (beta <= tolerance) converged = 1;
	}
	if (residual_out) *residual_out = residual;
	free(inverse); free(raw); free(res); free(work); free(V); free(h); free(cs); free(sn); free(g); free(y);
	return converged ? iterations : TFO_NOT_CONVERGED;
}

int tfo_gmres_bjacobi(int nodes, const int* row_offsets, const int* columns, const int* diagonal,
	const double* values, const double* rhs, double* x, int restart, int maximum_iterations,
	double rtol, double* residual_out, int* singular_out)
{
	return gmres_precond_f(4, nodes, row_offsets, columns, diagonal, values, rhs, x, restart, maximum_iterations,
		rtol, residual_out, singular_out, NULL, NULL);
}

/* The same GMRES on the 2x2 transport system (SolveGmres<2>, iga_cuda.cu:691). */
int tfo_transport_gmres(int nodes, const int* row_offsets, const int* columns, const int* diagonal,
	const double* values, const double* rhs, double* x, int restart, int maximum_iterations,
	double rtol, double* residual_out, int* singular_out)
{
	return gmres_precond_f(2, nodes, row_offsets, columns, diagonal, values, rhs, x, restart, maximum_iterations,
		rtol, residual_out, singular_out, NULL, NULL);
}

/* y = A x over 2x2 blocks (BlockSpmvKernel<2>). */
void tfo_transport_spmv(int nodes, const int* row_offsets, const int* columns, const double* values,
	const double* x, double* y)
{
	spmv_f(2, nodes, row_offsets, columns, values, x, y);
}

/*
 * Flow-line preconditioner for the 2x2 transport system (no counterpart in the reference, which
 * uses block-Jacobi): the restatement a device version is checked against.
 *
 * Lines: node i links to the pattern neighbour j with the largest a_ij = L++_ji - L++_ij > 0
 * (the antisymmetric part of the advected species' block, positive towards downstream); a node
 * keeps only its strongest upstream link; every node without an upstream link starts a chain.
 * line_offsets[lines+1], line_nodes[nodes] (every node exactly once, in chain order).
 */
int tfo_flow_lines(int nodes, const int* row_offsets, const int* columns, const double* values, int* line_offsets,
	int* line_nodes)
{
	int* down = (int*)malloc(sizeof(int)*(size_t)nodes);
	double* dval = (double*)malloc(sizeof(double)*(size_t)nodes);
	int* up = (int*)malloc(sizeof(int)*(size_t)nodes);
	double* uval = (double*)malloc(sizeof(double)*(size_t)nodes);
	char* seen = (char*)calloc((size_t)nodes, 1);
	if (!down || !dval || !up || !uval || !seen) return TFO_NO_MEMORY;
	for (int i = 0; i < nodes; ++i) {
		down[i] = -1; dval[i] = 0.0; up[i] = -1; uval[i] = 0.0;
		for (int b = row_offsets[i]; b < row_offsets[i+1]; ++b) {
			const int j = columns[b];
			if (j == i) continue;
			const long long t = find_block(row_offsets, columns, j, i);
			const double a = (t >= 0 ? values[t*4+3] : 0.0)-values[(size_t)b*4+3];
			if (a > dval[i]) { dval[i] = a; down[i] = j; }
		}
	}
	for (int i = 0; i < nodes; ++i) {
		const int j = down[i];
		if (j >= 0 && (up[j] < 0 || dval[i] > uval[j])) { up[j] = i; uval[j] = dval[i]; }
	}
	for (int i = 0; i < nodes; ++i)
		if (down[i] >= 0 && up[down[i]] != i) down[i] = -1;
	int lines = 0, at = 0;
	line_offsets[0] = 0;
	for (int h = 0; h < nodes; ++h) {
		if (up[h] >= 0 || seen[h]) continue;
		for (int i = h; i >= 0 && !seen[i]; i = down[i]) { seen[i] = 1; line_nodes[at++] = i; }
		line_offsets[++lines] = at;
	}
	/* nodes on closed loops (every node has an upstream link): each loop becomes one line */
	for (int h = 0; h < nodes; ++h) {
		if (seen[h]) continue;
		for (int i = h; i >= 0 && !seen[i]; i = down[i]) { seen[i] = 1; line_nodes[at++] = i; }
		line_offsets[++lines] = at;
	}
	free(down); free(dval); free(up); free(uval); free(seen);
	return lines;
}

/* 2x2 helpers (row-major). */
static void inv2(const double* a, double* r)
{
	const double det = a[0]*a[3]-a[1]*a[2];
	r[0] = a[3]/det; r[1] = -a[1]/det; r[2] = -a[2]/det; r[3] = a[0]/det;
}
static void mul2(const double* a, const double* b, double* r)
{
	r[0] = a[0]*b[0]+a[1]*b[2]; r[1] = a[0]*b[1]+a[1]*b[3];
	r[2] = a[2]*b[0]+a[3]*b[2]; r[3] = a[2]*b[1]+a[3]*b[3];
}

/*
 * Banded block LU (no pivoting) of every line's 2x2-block submatrix.  band_width[line] = the
 * largest |position difference| of two coupled nodes of the line; band_offsets[line] = start of
 * its storage in `factors` (4 doubles per block, m rows of 2w+1 blocks, block (p, q) at
 * row p, slot q - p + w).  Returns the number of doubles `factors` needs when factors == NULL.
 * After the call the band holds L (unit lower, below the diagonal) and U (on and above it), and
 * the diagonal slots hold U_pp^{-1}.
 */
long long tfo_line_factors(int nodes, const int* row_offsets, const int* columns, const double* values,
	int lines, const int* line_offsets, const int* line_nodes, int* band_width, long long* band_offsets,
	double* factors)
{
	int* pos = (int*)malloc(sizeof(int)*(size_t)nodes);
	int* line_of = (int*)malloc(sizeof(int)*(size_t)nodes);
	if (!pos || !line_of) return TFO_NO_MEMORY;
	for (int l = 0; l < lines; ++l)
		for (int k = line_offsets[l]; k < line_offsets[l+1]; ++k) {
			pos[line_nodes[k]] = k-line_offsets[l];
			line_of[line_nodes[k]] = l;
		}
	long long total = 0;
	for (int l = 0; l < lines; ++l) {
		int w = 0;
		for (int k = line_offsets[l]; k < line_offsets[l+1]; ++k) {
			const int i = line_nodes[k];
			for (int b = row_offsets[i]; b < row_offsets[i+1]; ++b)
				if (line_of[columns[b]] == l) {
					const int d = abs(pos[columns[b]]-pos[i]);
					if (d > w) w = d;
				}
		}
		band_width[l] = w;
		band_offsets[l] = total;
		total += 4LL*(line_offsets[l+1]-line_offsets[l])*(2*w+1);
	}
	if (!factors) { free(pos); free(line_of); return total; }
	memset(factors, 0, sizeof(double)*(size_t)total);
	for (int l = 0; l < lines; ++l) {
		const int m = line_offsets[l+1]-line_offsets[l], w = band_width[l], s = 2*w+1;
		double* B = factors+band_offsets[l];
		for (int k = line_offsets[l]; k < line_offsets[l+1]; ++k) {
			const int i = line_nodes[k], p = pos[i];
			for (int b = row_offsets[i]; b < row_offsets[i+1]; ++b)
				if (line_of[columns[b]] == l)
					memcpy(B+4*((size_t)p*s+(pos[columns[b]]-p+w)), values+(size_t)b*4, 4*sizeof(double));
		}
		for (int p = 0; p < m; ++p) {
			double dinv[4], lrp[4], t[4];
			inv2(B+4*((size_t)p*s+w), dinv);
			for (int r = p+1; r <= p+w && r < m; ++r) {
				double* Arp = B+4*((size_t)r*s+(p-r+w));
				mul2(Arp, dinv, lrp);
				memcpy(Arp, lrp, sizeof(lrp));
				for (int c = p+1; c <= p+w && c < m; ++c) {
					double* Arc = B+4*((size_t)r*s+(c-r+w));
					mul2(lrp, B+4*((size_t)p*s+(c-p+w)), t);
					for (int e = 0; e < 4; ++e) Arc[e] -= t[e];
				}
			}
			memcpy(B+4*((size_t)p*s+w), dinv, sizeof(dinv));
		}
	}
	free(pos); free(line_of);
	return total;
}

/* out = M^{-1} in: forward and backward substitution along every line. */
void tfo_line_apply(int lines, const int* line_offsets, const int* line_nodes, const int* band_width,
	const long long* band_offsets, const double* factors, const double* in, double* out)
{
#pragma omp parallel for schedule(dynamic, 16)
	for (int l = 0; l < lines; ++l) {
		const int m = line_offsets[l+1]-line_offsets[l], w = band_width[l], s = 2*w+1;
		const double* B = factors+band_offsets[l];
		const int* nodes = line_nodes+line_offsets[l];
		double* y = (double*)malloc(sizeof(double)*2*(size_t)m);
		for (int p = 0; p < m; ++p) {
			double v0 = in[2*(size_t)nodes[p]], v1 = in[2*(size_t)nodes[p]+1];
			for (int q = p-w > 0 ? p-w : 0; q < p; ++q) {
				const double* L = B+4*((size_t)p*s+(q-p+w));
				v0 -= L[0]*y[2*q]+L[1]*y[2*q+1];
				v1 -= L[2]*y[2*q]+L[3]*y[2*q+1];
			}
			y[2*p] = v0; y[2*p+1] = v1;
		}
		for (int p = m-1; p >= 0; --p) {
			double v0 = y[2*p], v1 = y[2*p+1];
			for (int q = p+1; q <= p+w && q < m; ++q) {
				const double* U = B+4*((size_t)p*s+(q-p+w));
				v0 -= U[0]*y[2*q]+U[1]*y[2*q+1];
				v1 -= U[2]*y[2*q]+U[3]*y[2*q+1];
			}
			const double* D = B+4*((size_t)p*s+w);
			y[2*p] = D[0]*v0+D[1]*v1;
			y[2*p+1] = D[2]*v0+D[3]*v1;
		}
		for (int p = 0; p < m; ++p) { out[2*(size_t)nodes[p]] = y[2*p]; out[2*(size_t)nodes[p]+1] = y[2*p+1]; }
		free(y);
	}
}

typedef struct {
	int lines;
	const int* line_offsets;
	const int* line_nodes;
	const int* band_width;
	const long long* band_offsets;
	const double* factors;
} line_context;

static void line_precond(const void* context, const double* in, double* out)
{
	const line_context* c = (const line_context*)context;
	tfo_line_apply(c->lines, c->line_offsets, c->line_nodes, c->band_width, c->band_offsets, c->factors, in, out);
}

/* GMRES(restart) on the 2x2 transport system, left-preconditioned with the flow-line factors. */
int tfo_transport_gmres_lines(int nodes, const int* row_offsets, const int* columns, const double* values,
	int lines, const int* line_offsets, const int* line_nodes, const int* band_width, const long long* band_offsets,
	const double* factors, const double* rhs, double* x, int restart, int maximum_iterations, double rtol,
	double* residual_out)
{
	const line_context c = {lines, line_offsets, line_nodes, band_width, band_offsets, factors};
	return gmres_precond_f(2, nodes, row_offsets, columns, NULL, values, rhs, x, restart, maximum_iterations, rtol,
		residual_out, NULL, line_precond, &c);
}

int tfo_max_threads(void)
{
#ifdef _OPENMP
	return omp_get_max_threads();
#else
	return 1;
#endif
}

/* ---------------------------------------------------------------------------
 * Two-species transport (N0 attached, N+ advected): the reference's
 * `iga_cuda transport` path.
 * ------------------------------------------------------------------------- */

/*
 * Transport parameters, in the order of iga::TransportParameters
 * (solvers/cpu/include/CaseInput.hpp:19-33): D, vplus, vminus, kplus,
 * kminus, k'plus, k'minus, dt, (steps), N0bc, Nplusbc, Nminusbc,
 * artificial_diffusion.  Only the ones the element reads are passed here:
 * p[0] D, p[1] vplus, p[2] kplus, p[3] kminus, p[4] k'plus, p[5] dt,
 * p[6] artificial_diffusion.
 */

/*
 * BuildTransportElement (TransportElement.hpp:213-253; the device form is
 * AssembleTransportKernel, IgaCudaKernels.cuh:155-237): the backward-Euler
 * left matrix and the previous-state matrix of one element, dense
 * (2 nen)^2 with dof 2a = N0 and 2a+1 = N+ of basis a.  velocity[a*3+d] is
 * the nodal velocity of basis a.  Per Gauss point:
 *   u = sum_a N_a u_a,  tau = (|u.grad N|_1^-2 + (dt/2)^-2)^-1/2 (0 if u.grad N = 0),
 *   T_a = N_a + tau u.grad N_a (SUPG test function of N+),
 *   L00 += ((1 + dt (k+ + k-)) N_a N_b + dt D grad N_a.grad N_b) w
 *   L0+ += -k'+ dt N_a N_b w
 *   L+0 += -k+ dt T_a N_b w
 *   L++ += ((1 + dt k'+) T_a N_b + dt T_a u.grad N_b + dt v+ ad T_a grad N_a.grad N_b) w
 *   P00 += N_a N_b w,  P++ += T_a N_b w,
 * with w the Gauss weight times det(dx/dxi).
 */
int tfo_transport_element(const double* C, const double* X, int nen, const double* velocity,
	const double* p, double* left, double* previous)
{
	if (nen <= 0 || nen > 80) return TFO_BAD_INPUT;
	const double D = p[0], vplus = p[1], kplus = p[2], kminus = p[3], detach = p[4], dt = p[5],
		artificial = p[6];
	const int ndof = 2*nen;
	memset(left, 0, sizeof(double)*(size_t)ndof*ndof);
	memset(previous, 0, sizeof(double)*(size_t)ndof*ndof);
	double qp[64*3], qw[64], N[80], dN[240], T[80], inv[9], det;
	tfo_gauss_rule(qp, qw);
	for (int q = 0; q < 64; ++q) {
		const int st = tfo_basis(C, X, nen, qp[3*q], qp[3*q+1], qp[3*q+2], 0, N, dN, NULL, inv, &det);
		if (st != TFO_OK) return st;
		const double w = qw[q]*det;
		double u[3] = {0.0, 0.0, 0.0};
		for (int a = 0; a < nen; ++a)
			for (int d = 0; d < 3; ++d) u[d] += N[a]*velocity[a*3+d];
		double inverse_length = 0.0;
		for (int a = 0; a < nen; ++a)
			inverse_length += fabs(u[0]*dN[3*a]+u[1]*dN[3*a+1]+u[2]*dN[3*a+2]);
		const double tau_space = inverse_length > 0.0 ? 1.0/inverse_length : 0.0;
		const double tau_time = dt/2.0;
		const double tau = tau_space > 0.0
			? 1.0/sqrt(1.0/(tau_space*tau_space)+1.0/(tau_time*tau_time)) : 0.0;
		for (int a = 0; a < nen; ++a)
			T[a] = N[a]+tau*(u[0]*dN[3*a]+u[1]*dN[3*a+1]+u[2]*dN[3*a+2]);
		for (int a = 0; a < nen; ++a)
			for (int b = 0; b < nen; ++b) {
				const double gg = dN[3*a]*dN[3*b]+dN[3*a+1]*dN[3*b+1]+dN[3*a+2]*dN[3*b+2];
				const double adv = u[0]*dN[3*b]+u[1]*dN[3*b+1]+u[2]*dN[3*b+2];
				const double mass = N[a]*N[b];
				double* l0 = left+(size_t)(2*a)*ndof+2*b;
				double* lp = left+(size_t)(2*a+1)*ndof+2*b;
				l0[0] += ((1.0+dt*(kplus+kminus))*mass+dt*D*gg)*w;
				l0[1] += -detach*dt*mass*w;
				lp[0] += -kplus*dt*T[a]*N[b]*w;
				lp[1] += ((1.0+dt*detach)*T[a]*N[b]+dt*T[a]*adv+dt*vplus*artificial*T[a]*gg)*w;
				previous[(size_t)(2*a)*ndof+2*b] += mass*w;
				previous[(size_t)(2*a+1)*ndof+2*b+1] += T[a]*N[b]*w;
			}
	}
	return TFO_OK;
}

/*
 * Global transport assembly into 2x2 block CSR (values[block*4 + 2i + j]) over
 * the node-graph pattern, then the boundary rows of ApplyTransportBoundaryKernel
 * (IgaCudaKernels.cuh:411-424): a constrained node's row blocks are zeroed in
 * both matrices and its diagonal block of `left` becomes the identity.
 * velocity[node*3+d]; constrained[node] != 0 marks a Dirichlet node (may be NULL).
 */
int tfo_transport_assemble(int nodes, int elements, const int* element_offsets, const int* connectivity,
	const int* extraction_offsets, const uint8_t* extraction_columns, const double* extraction_values,
	const double* bezier_points, const int* row_offsets, const int* columns, const int* diagonal,
	const double* velocity, const double* p, const int* constrained, double* left, double* previous,
	int* failed_element)
{
	int failure = -1, status_out = TFO_OK;
#pragma omp parallel
	{
		double* C = (double*)malloc(sizeof(double)*80*64);
		double* el = (double*)malloc(sizeof(double)*160*160);
		double* ep = (double*)malloc(sizeof(double)*160*160);
		double vel[240];
		long long blocks[80];
#pragma omp for schedule(dynamic, 4)
		for (int e = 0; e < elements; ++e) {
			const int begin = element_offsets[e];
			const int nen = element_offsets[e+1]-begin;
			memset(C, 0, sizeof(double)*(size_t)nen*64);
			for (int a = 0; a < nen; ++a) {
				for (int k = extraction_offsets[begin+a]; k < extraction_offsets[begin+a+1]; ++k)
					C[a*64+extraction_columns[k]] = extraction_values[k];
				for (int d = 0; d < 3; ++d) vel[a*3+d] = velocity[3*(size_t)connectivity[begin+a]+d];
			}
			const int status = tfo_transport_element(C, bezier_points+(size_t)e*192, nen, vel, p, el, ep);
			if (status != TFO_OK) {
#pragma omp critical
				{ failure = e; status_out = status; }
				continue;
			}
			const int ndof = 2*nen;
			for (int a = 0; a < nen; ++a) {
				const int row = connectivity[begin+a];
				for (int b = 0; b < nen; ++b)
					blocks[b] = find_block(row_offsets, columns, row, connectivity[begin+b]);
				for (int b = 0; b < nen; ++b)
					for (int i = 0; i < 2; ++i)
						for (int j = 0; j < 2; ++j) {
							const size_t at = (size_t)(2*a+i)*ndof+2*b+j;
#pragma omp atomic
							left[blocks[b]*4+2*i+j] += el[at];
#pragma omp atomic
							previous[blocks[b]*4+2*i+j] += ep[at];
						}
			}
		}
		free(C); free(el); free(ep);
	}
	if (failed_element) *failed_element = failure;
	if (status_out != TFO_OK || !constrained) return status_out;
	for (int node = 0; node < nodes; ++node) {
		if (!constrained[node]) continue;
		for (int b = row_offsets[node]; b < row_offsets[node+1]; ++b)
			for (int k = 0; k < 4; ++k) { left[(size_t)b*4+k] = 0.0; previous[(size_t)b*4+k] = 0.0; }
		left[(size_t)diagonal[node]*4] = 1.0;
		left[(size_t)diagonal[node]*4+3] = 1.0;
	}
	return TFO_OK;
}
