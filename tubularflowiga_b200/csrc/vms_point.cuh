// Per-quadrature-point VMS Navier-Stokes quantities shared by the FP64
// assembly kernel and the tensor-core tangent kernel.
//
// Formulation: the reference's BuildNavierStokesElementFromPreparedPoints
// (solvers/cpu/include/NavierStokesElement.hpp:149-317, LegacyBodyFitted weak
// form, zero body force), with the exact Newton tangent (:244-312).  At each
// point every tangent term is a product (test feature s of N_a) x (trial
// feature t of N_b), s in {N, dN/dx, dN/dy, dN/dz}, t in {N, dN/dx, dN/dy,
// dN/dz, Lap N}; RowCoefficients collects those products per (row field i,
// column field f).
#pragma once

#include "kernels.cuh"

namespace tfiga {

constexpr int kQS = 24;                         // per-point state slots in shared memory
constexpr int kCoef = 80;                       // 4 f x 4 s x 5 t tangent coefficients

// Per-point state slots.
enum : int { kU = 0, kP = 3, kUp = 4, kGrad = 7 /* 12: du_f/dx_d at 7+3f+d, f=3: pressure */, kLap = 19 };

struct PointState {
	double u[3], p, up[3], gv[3][3], gp[3], lap[3];
};

// Coefficients of row field i at one point, all scaled by the point
// measure: M[((f - f_lo)*20 + s*5 + t)*kStride] multiplies (test feature s
// of N_a) x (trial feature t of N_b) in K^{if}_{ab}; rc[s] = -measure * c_s
// gives the residual.  Computed in FP64; C is the storage type of M (double
// for the FP64 tangent, float for the tensor-core tangent).  Only the column
// fields f in [f_lo, f_hi) are written; rc may be null.  kTangent false: only
// rc is computed (M is not touched and may be null).
template <class C, int kStride = 1, bool kTangent = true>
__device__ __forceinline__ void RowCoefficients(int i, const PointState& S, const double* qd,
	const AssemblyParams& prm, C* M, double* rc, int f_lo = 0, int f_hi = 4)
{
	const double rho = prm.density, mu = prm.viscosity, nu = mu/rho;
	const double dt = prm.dt;
	const double idt = dt > 0.0 ? 1.0/dt : 0.0;
	const double meas = qd[0];
	double G[3][3];
	G[0][0] = qd[1]; G[0][1] = G[1][0] = qd[2]; G[0][2] = G[2][0] = qd[3];
	G[1][1] = qd[4]; G[1][2] = G[2][1] = qd[5]; G[2][2] = qd[6];
	const double dnorm = qd[7], gnorm = qd[8];
	double dudt[3];
	for (int c = 0; c < 3; ++c) dudt[c] = dt > 0.0 ? (S.u[c]-S.up[c])/dt : 0.0;
	// Stabilization (NavierStokesElement.hpp:121-144).
	double Gu[3], vm = 0.0;
	for (int f = 0; f < 3; ++f) {
		Gu[f] = G[f][0]*S.u[0]+G[f][1]*S.u[1]+G[f][2]*S.u[2];
		vm += S.u[f]*Gu[f];
	}
	const double temporal = dt > 0.0 ? 4.0*idt*idt : 0.0;
	const double tau_m = 1.0/sqrt(temporal+vm+(1.0/12.0)*nu*nu*gnorm);
	const double tau_c = 1.0/(tau_m*dnorm);
	// Strong residual, fine-scale velocity and pressure (:202-211).
	double R[3], fine[3], a[3];
	for (int c = 0; c < 3; ++c) {
		R[c] = dudt[c]+S.u[0]*S.gv[c][0]+S.u[1]*S.gv[c][1]+S.u[2]*S.gv[c][2]+S.gp[c]/rho-nu*S.lap[c];
		fine[c] = -tau_m*R[c];
		a[c] = S.u[c]+fine[c];
	}
	const double divu = S.gv[0][0]+S.gv[1][1]+S.gv[2][2];
	const double fine_p = -rho*tau_c*divu;
	// Residual (:218-239).
	if (rc == nullptr) {
	} else if (i < 3) {
		double cN = rho*dudt[i];
		for (int d = 0; d < 3; ++d) cN += rho*a[d]*S.gv[i][d];
		rc[0] = -meas*cN;
		for (int d = 0; d < 3; ++d) {
			double cd = mu*(S.gv[i][d]+S.gv[d][i])-rho*fine[i]*a[d];
			if (d == i) cd -= S.p+fine_p;
			rc[1+d] = -meas*cd;
		}
	} else {
		rc[0] = -meas*divu;
		for (int d = 0; d < 3; ++d) rc[1+d] = meas*fine[d];
	}
	if constexpr (!kTangent) return;
	// Exact tangent (:248-312), collected by (test, trial) feature.
	const double t3 = tau_m*tau_m*tau_m;
	double dtau_c[3], A[3][3];
	for (int f = 0; f < 3; ++f) {
		const double dtau_m = -t3*Gu[f];
		dtau_c[f] = tau_c*tau_m*tau_m*Gu[f];
		for (int c = 0; c < 3; ++c)
			A[c][f] = -dtau_m*R[c]-tau_m*((c == f ? idt : 0.0)+S.gv[c][f]);
	}
	for (int k = 0; k < (f_hi-f_lo)*20; ++k) M[k*kStride] = C(0);
	auto at = [&](int f, int s, int t) -> C& { return M[((f-f_lo)*20+s*5+t)*kStride]; };
	const int f_vel = f_hi < 3 ? f_hi : 3;     // end of the velocity columns in range
	const bool p_col = f_hi > 3;               // pressure column in range
	if (i < 3) {
		for (int f = f_lo; f < f_vel; ++f) {
			double nn = rho*S.gv[i][f]+(f == i ? rho*idt : 0.0);
			for (int d = 0; d < 3; ++d) nn += rho*A[d][f]*S.gv[i][d];
			at(f, 0, 0) = nn;
			for (int e = 0; e < 3; ++e) at(f, 0, 1+e) = -rho*tau_m*S.gv[i][f]*S.u[e]+(f == i ? rho*a[e] : 0.0);
			at(f, 0, 4) = rho*tau_m*nu*S.gv[i][f];
			for (int d = 0; d < 3; ++d) {
				at(f, 1+d, 0) = (d == i ? rho*dtau_c[f]*divu : 0.0)-rho*a[d]*A[i][f]
					-rho*fine[i]*((d == f ? 1.0 : 0.0)+A[d][f]);
				for (int e = 0; e < 3; ++e) {
					double v = 0.0;
					if (d == i && e == f) v += rho*tau_c;
					if (f == i && d == e) v += mu;
					if (f == d && e == i) v += mu;
					if (f == i) v += rho*tau_m*a[d]*S.u[e];
					if (d == f) v += rho*tau_m*fine[i]*S.u[e];
					at(f, 1+d, 1+e) = v;
				}
				at(f, 1+d, 4) = -rho*tau_m*nu*((f == i ? a[d] : 0.0)+(d == f ? fine[i] : 0.0));
			}
		}
		if (p_col) {
			at(3, 1+i, 0) = -1.0;
			for (int e = 0; e < 3; ++e) at(3, 0, 1+e) = -tau_m*S.gv[i][e];
			for (int d = 0; d < 3; ++d)
				for (int e = 0; e < 3; ++e)
					at(3, 1+d, 1+e) = tau_m*((e == i ? a[d] : 0.0)+(d == e ? fine[i] : 0.0));
		}
	} else {
		for (int f = f_lo; f < f_vel; ++f) {
			at(f, 0, 1+f) = 1.0;
			for (int d = 0; d < 3; ++d) at(f, 1+d, 0) = -A[d][f];
			for (int e = 0; e < 3; ++e) at(f, 1+f, 1+e) = tau_m*S.u[e];
			at(f, 1+f, 4) = -tau_m*nu;
		}
		if (p_col)
			for (int d = 0; d < 3; ++d) at(3, 1+d, 1+d) = tau_m/rho;
	}
	for (int k = 0; k < (f_hi-f_lo)*20; ++k) M[k*kStride] = C(M[k*kStride]*meas);
}

} // namespace tfiga
