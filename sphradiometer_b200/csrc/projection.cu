// projection.cu -- the projection operator of the inspiral path multiplied
// into a baseline's delay kernel, every frequency bin at once on the GPU.
//
// The reference (correlator_network_plan_mult_by_projection,
// inspiral_sky_map.c:423-549, with correlator_plan_mult_by_projection,
// :387-420) builds, for each baseline (a, b) and frequency bin j, the
// function on the sky
//     P_ab(theta, phi) = u_a conj(u_b) / sum_k |u_k|^2 - delta_ab,
//     u_k = (F+_k + i beta Fx_k) / S_j,k          (CBCProjectionMatrix, :342-364,
//                                                  |u_k|^2 as F+^2 + beta^2 Fx^2)
// projects it onto spherical harmonics on its mesh (sh_series_from_func),
// rotates it into the baseline frame (sh_series_invrot_matrix) and
// multiplies it into the bin's polar delay kernel (sh_series_product),
// one bin at a time on the CPU.  Here the antenna patterns come in once,
// sampled on the same mesh, and a chunk of bins goes through four
// batched stages: the mesh of every bin's P (k_projection_mesh), the
// analysis transform, the rotation and the pixel-domain product.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "runtime.h"

namespace sphrad {

namespace {

__global__ void k_projection_mesh(const double *__restrict__ fp, const double *__restrict__ fc, int n_det, int npix, const double *__restrict__ psd, int j0, int nb,
				  int a, int b, double beta, double2 *__restrict__ mesh)
{
	const long long total = (long long) nb * npix;
	for(long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < total; i += (long long) gridDim.x * blockDim.x) {
		const int j = (int) (i / npix), p = (int) (i - (long long) j * npix);
		const double *S = psd + (size_t) (j0 + j) * n_det;
		double norm = 0.0;
		for(int k = 0; k < n_det; k++) {
			const double x = fp[(size_t) k * npix + p] / S[k], y = fc[(size_t) k * npix + p] / S[k];
			norm += x * x + beta * beta * y * y;
		}
		const double xa = fp[(size_t) a * npix + p] / S[a], ya = beta * fc[(size_t) a * npix + p] / S[a];
		const double xb = fp[(size_t) b * npix + p] / S[b], yb = beta * fc[(size_t) b * npix + p] / S[b];
		// (xa + i ya)(xb - i yb) / norm - delta_ab
		double re = (xa * xb + ya * yb) / norm, im = (ya * xb - xa * yb) / norm;
		if(a == b)
			re -= 1.0;
		mesh[i] = make_double2(re, im);
	}
}

struct DevBuf {
	void *p = nullptr;
	explicit DevBuf(size_t bytes) { p = dmalloc(bytes ? bytes : 16); }
	~DevBuf() { dfree(p); }
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
};

}  // namespace

int projection_multiply(int n, unsigned L, int n_det, const double *fp_host, const double *fc_host, const double *psd_host, int a, int b, double beta,
			const double *Rinv, const double *delay_host, double *out_host)
{
	if(ensure_device())
		return -1;
	if(n <= 0 || n_det < 2 || a < 0 || b < 0 || a >= n_det || b >= n_det) {
		set_error("projection: bad bins (%d), detectors (%d) or baseline (%d, %d)", n, n_det, a, b);
		return -1;
	}
	const int nt = 2 * ((int) L + 1), np = nt, npix = nt * np;
	const size_t nq = (size_t) (L + 1) * (L + 1), np1 = (size_t) L + 1;
	// the reference's mesh for the projection; a grid that integrates the
	// product's degree 3L exactly for the multiplication
	void *mesh_plan = sht_plan_create(L, kGridGL, nt, np, 0);
	void *prod_plan = sht_plan_create(L, kGridGL, (int) (3 * L) / 2 + 1, (int) (3 * L) + 1, 0);
	int rc = -1;
	const int chunk = n < 512 ? n : 512;
	{
		DevBuf dfp((size_t) n_det * npix * 8), dfc((size_t) n_det * npix * 8), dpsd((size_t) n * n_det * 8), dR((size_t) chunk * 9 * 8),
			dmesh((size_t) chunk * npix * 16), dcoef((size_t) chunk * nq * 16), drot((size_t) chunk * nq * 16), ddel((size_t) chunk * np1 * 16),
			dout((size_t) chunk * nq * 16);
		const size_t s_an = mesh_plan ? sht_scratch_bytes(mesh_plan, chunk, (int) L) : 0;
		const size_t s_rot = rotate_batch_scratch_bytes(L, chunk);
		const size_t s_pr = prod_plan ? sht_product_scratch_bytes(prod_plan, chunk, L, 1, L, 0, L, 0) : 0;
		DevBuf dscr(s_an > s_rot ? (s_an > s_pr ? s_an : s_pr) : (s_rot > s_pr ? s_rot : s_pr));
		std::vector<double> Rrep((size_t) chunk * 9);
		for(int i = 0; i < chunk; i++)
			for(int k = 0; k < 9; k++)
				Rrep[(size_t) i * 9 + k] = Rinv[k];
		bool ok = mesh_plan && prod_plan && dfp.p && dfc.p && dpsd.p && dR.p && dmesh.p && dcoef.p && drot.p && ddel.p && dout.p && dscr.p &&
			  !h2d(dfp.p, fp_host, (size_t) n_det * npix * 8) && !h2d(dfc.p, fc_host, (size_t) n_det * npix * 8) &&
			  !h2d(dpsd.p, psd_host, (size_t) n * n_det * 8) && !h2d(dR.p, Rrep.data(), Rrep.size() * 8);
		void *st = lib_stream();
		const size_t scr_bytes = s_an > s_rot ? (s_an > s_pr ? s_an : s_pr) : (s_rot > s_pr ? s_rot : s_pr);
		for(int j0 = 0; ok && j0 < n; j0 += chunk) {
			const int c = n - j0 < chunk ? n - j0 : chunk;
			k_projection_mesh<<<592, 256, 0, (cudaStream_t) st>>>((const double *) dfp.p, (const double *) dfc.p, n_det, npix, (const double *) dpsd.p, j0,
									     c, a, b, beta, (double2 *) dmesh.p);
			ok = cudaGetLastError() == cudaSuccess && !h2d(ddel.p, delay_host + (size_t) j0 * np1 * 2, (size_t) c * np1 * 16) &&
			     !sht_analysis(mesh_plan, dmesh.p, c, L, 0, dcoef.p, (long long) nq, dscr.p, st) &&
			     !rotate_batch(dcoef.p, c, L, 0, (const double *) dR.p, drot.p, 0, dscr.p, scr_bytes, st) &&
			     !sht_product(prod_plan, c, ddel.p, (long long) np1, L, 1, drot.p, (long long) nq, L, 0, dout.p, (long long) nq, L, 0, dscr.p, st) &&
			     !d2h(out_host + (size_t) j0 * nq * 2, dout.p, (size_t) c * nq * 16) && !stream_sync();
			if(!ok)
				set_error("projection: GPU stage failed at bins %d..%d", j0, j0 + c - 1);
		}
		rc = ok ? 0 : -1;
	}
	sht_plan_destroy(mesh_plan);
	sht_plan_destroy(prod_plan);
	return rc;
}

}  // namespace sphrad

// ------------------------------------------------------------------------
// projection matrix of an off-axis phase centre (projection.c:99-131): each
// tap's sinc(pi (-k - r.s / dt)) is sampled on the reference's mesh of
// l_max L and analysed, a chunk of taps per batched transform
// ------------------------------------------------------------------------
namespace sphrad {

namespace {

__global__ void k_delay_mesh(const double *__restrict__ theta, int nt, int nphi, double rx, double ry, double rz, double dt, int k0, int nb,
			     double2 *__restrict__ mesh)
{
	const long long npix = (long long) nt * nphi, total = (long long) nb * npix;
	for(long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < total; i += (long long) gridDim.x * blockDim.x) {
		const int c = (int) (i / npix);
		const long long p = i - (long long) c * npix;
		const int it = (int) (p / nphi), jp = (int) (p - (long long) it * nphi);
		double st, ct, sp, cp;
		sincos(theta[it], &st, &ct);
		sincospi(2.0 * jp / nphi, &sp, &cp);
		const double rs = rx * st * cp + ry * st * sp + rz * ct;
		const double pi_x = M_PI * (0 - (k0 + c) - rs / dt);
		mesh[i] = make_double2(pi_x == 0.0 ? 1.0 : sin(pi_x) / pi_x, 0.0);
	}
}

}  // namespace

int projection_taps_full(const double *r, double delta_t, int n_el, unsigned L, double *series_host)
{
	if(!(delta_t > 0) || n_el <= 0) {
		set_error("projection matrix: bad sample interval %g or %d taps", delta_t, n_el);
		return -1;
	}
	if(ensure_device())
		return -1;
	const int nt = 2 * ((int) L + 1), nphi = nt;
	const size_t len = (size_t) (L + 1) * (L + 1), npix = (size_t) nt * nphi;
	void *plan = sht_plan_create(L, kGridGL, nt, nphi, 0);
	if(!plan)
		return -1;
	int chunk = (int) std::max<size_t>(1, std::min<size_t>((size_t) 256 << 20, (size_t) 64 * npix * 16) / (npix * 16));
	if(chunk > n_el)
		chunk = n_el;
	int rc = -1;
	{
		const size_t scr = sht_scratch_bytes(plan, chunk, (int) L);
		DevBuf dmesh((size_t) chunk * npix * 16), dout((size_t) chunk * len * 16), dscr(scr);
		bool ok = dmesh.p && dout.p && dscr.p;
		void *st = lib_stream();
		const int k_first = -(n_el - 1) / 2;
		for(int t0 = 0; ok && t0 < n_el; t0 += chunk) {
			const int c = n_el - t0 < chunk ? n_el - t0 : chunk;
			k_delay_mesh<<<592, 256, 0, (cudaStream_t) st>>>(sht_plan_theta_dev(plan), nt, nphi, r[0], r[1], r[2], delta_t, k_first + t0, c,
									   (double2 *) dmesh.p);
			ok = cudaGetLastError() == cudaSuccess && !sht_analysis(plan, dmesh.p, c, L, 0, dout.p, (long long) len, dscr.p, st) &&
			     !d2h(series_host + (size_t) t0 * len * 2, dout.p, (size_t) c * len * 16) && !stream_sync();
			if(!ok)
				set_error("projection matrix: GPU stage failed at taps %d..%d", t0, t0 + c - 1);
		}
		rc = ok ? 0 : -1;
	}
	sht_plan_destroy(plan);
	return rc;
}

}  // namespace sphrad
