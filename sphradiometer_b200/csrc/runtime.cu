// runtime.cu -- device context and the FP64 kernels of the drop-in path:
// delay-table (D_l(k)) construction, Wigner-D rotation plans, rotation,
// and the per-call frequency-domain integrator.
//
// Reference algorithms (cannon-zz/sphradiometer):
//   delay table      correlator.c:424-519, projection.c:99-131,
//                    sh_series_trans.c:663-734, sh_series_product.c:269-329
//   rotation plan    sh_series_rotation.c:279-422 (Choi, Ivanic, Gordon &
//                    Ruedenberg recursion)
//   rotation         sh_series_rotation.c:546-589
//   integration      correlator.c:681-711 and 993-1010
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "runtime.h"
#include "wigner.cuh"

namespace sphrad {

// ------------------------------------------------------------------------
// errors
// ------------------------------------------------------------------------
static thread_local std::string g_err;

void set_error(const char *fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	g_err = buf;
}

const char *last_error() { return g_err.c_str(); }

#define CK(call)                                                                 \
	do {                                                                     \
		cudaError_t e_ = (call);                                         \
		if(e_ != cudaSuccess) {                                          \
			set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
			return -1;                                               \
		}                                                                \
	} while(0)

// ------------------------------------------------------------------------
// device context: one non-blocking stream per device
// ------------------------------------------------------------------------
static std::mutex g_ctx_mu;
static std::unordered_map<int, cudaStream_t> g_streams;
// per device, a stream-ordered memory pool for the scratch of the
// synchronous drop-in calls, which keeps what it has allocated: a call
// takes and returns its scratch without cudaMalloc / cudaFree (whose free
// synchronises the whole device)
static std::unordered_map<int, cudaMemPool_t> g_pools;

int ensure_device()
{
	int n = 0;
	cudaError_t e = cudaGetDeviceCount(&n);
	if(e != cudaSuccess || n == 0) {
		set_error("no usable CUDA device (%s)", e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
		return -1;
	}
	int dev = 0;
	CK(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lk(g_ctx_mu);
	if(!g_streams.count(dev)) {
		cudaStream_t s;
		CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
		g_streams[dev] = s;
	}
	if(!g_pools.count(dev)) {
		cudaMemPoolProps props;
		memset(&props, 0, sizeof(props));
		props.allocType = cudaMemAllocationTypePinned;
		props.handleTypes = cudaMemHandleTypeNone;
		props.location.type = cudaMemLocationTypeDevice;
		props.location.id = dev;
		cudaMemPool_t pool;
		CK(cudaMemPoolCreate(&pool, &props));
		uint64_t keep = ~0ull;
		CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
		g_pools[dev] = pool;
	}
	return 0;
}

int current_device()
{
	int dev = 0;
	cudaGetDevice(&dev);
	return dev;
}

void *lib_stream()
{
	int dev = 0;
	cudaGetDevice(&dev);
	std::lock_guard<std::mutex> lk(g_ctx_mu);
	auto it = g_streams.find(dev);
	return it == g_streams.end() ? nullptr : (void *) it->second;
}

static cudaStream_t S() { return (cudaStream_t) lib_stream(); }

int sync_stream(void *stream)
{
	CK(cudaStreamSynchronize(stream ? (cudaStream_t) stream : S()));
	CK(cudaGetLastError());
	return 0;
}

int stream_sync()
{
	CK(cudaStreamSynchronize(S()));
	CK(cudaGetLastError());
	return 0;
}

static std::atomic<long> g_alloc_fault{0};

int set_alloc_fault(long n)
{
	g_alloc_fault.store(n > 0 ? n : 0);
	return 0;
}

bool alloc_fault_due()
{
	long v = g_alloc_fault.load();
	while(v > 0) {
		if(g_alloc_fault.compare_exchange_weak(v, v - 1))
			return v == 1;
	}
	return false;
}

void *dmalloc(size_t bytes)
{
	if(alloc_fault_due()) {
		set_error("cudaMalloc(%zu): injected allocation failure", bytes);
		return nullptr;
	}
	void *p = nullptr;
	cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
	if(e != cudaSuccess) {
		set_error("cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
		return nullptr;
	}
	return p;
}

void dfree(void *p)
{
	if(p)
		cudaFree(p);
}

void *dscratch(size_t bytes) { return dscratch_on(bytes, nullptr); }

void dscratch_free(void *p) { dscratch_free_on(p, nullptr); }

void *dscratch_on(size_t bytes, void *stream)
{
	if(alloc_fault_due()) {
		set_error("scratch of %zu bytes: injected allocation failure", bytes);
		return nullptr;
	}
	if(ensure_device())
		return nullptr;
	const int dev = current_device();
	cudaMemPool_t pool;
	{
		std::lock_guard<std::mutex> lk(g_ctx_mu);
		pool = g_pools[dev];
	}
	void *p = nullptr;
	cudaError_t e = cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, stream ? (cudaStream_t) stream : S());
	if(e != cudaSuccess) {
		set_error("scratch of %zu bytes: %s", bytes, cudaGetErrorString(e));
		return nullptr;
	}
	return p;
}

void dscratch_free_on(void *p, void *stream)
{
	if(p)
		cudaFreeAsync(p, stream ? (cudaStream_t) stream : S());
}

int h2d(void *dst, const void *src, size_t bytes)
{
	CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S()));
	return 0;
}

int d2h(void *dst, const void *src, size_t bytes)
{
	CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S()));
	return 0;
}

int dmemset_async(void *dst, int value, size_t bytes, void *stream)
{
	CK(cudaMemsetAsync(dst, value, bytes, stream ? (cudaStream_t) stream : S()));
	return 0;
}

int dmemset(void *dst, int value, size_t bytes)
{
	CK(cudaMemsetAsync(dst, value, bytes, S()));
	return 0;
}

// RAII device buffer
struct DBuf {
	void *p = nullptr;
	DBuf() = default;
	explicit DBuf(size_t bytes) { p = dscratch(bytes); }
	~DBuf() { dscratch_free(p); }
	DBuf(const DBuf &) = delete;
	DBuf &operator=(const DBuf &) = delete;
	template <class T> T *as() const { return (T *) p; }
};

// ------------------------------------------------------------------------
// small device helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }  // a * conj(b)

// sizing of the projection matrices: projection.c:56-87, correlator.c:55-65
static int n_elements(double r, double dt) { return 2 * (int) (60 + r / dt + 1) + 1; }
static unsigned proj_l_max(double r, double dt) { return (int) (M_PI * r / dt + 1); }
static unsigned power_l_max_naive(double d, double dt) { return (unsigned) floor(M_PI / (2. * asin(dt / (2. * d))) + 1.); }

// ------------------------------------------------------------------------
// Gauss-Legendre nodes (Newton on P_n), decreasing x  (the mesh ordering of
// sh_series_trans.c:149-196)
// ------------------------------------------------------------------------
__device__ static void legendre_pn(int n, double z, double *pn, double *pn1)
{
	double p0 = 1.0, p1 = z;
	for(int k = 2; k <= n; k++) {
		const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
		p0 = p1;
		p1 = p2;
	}
	*pn = p1;
	*pn1 = p0;
}

__global__ void k_gl_nodes(int n, double *x, double *w)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= (n + 1) / 2)
		return;
	double z = cos(M_PI * (i + 0.75) / (n + 0.5));
	double pn, pn1, pp = 1.0;
	for(int it = 0; it < 100; it++) {
		legendre_pn(n, z, &pn, &pn1);
		pp = n * (z * pn - pn1) / (z * z - 1.0);
		const double dz = pn / pp;
		z -= dz;
		if(fabs(dz) < 1e-16)
			break;
	}
	legendre_pn(n, z, &pn, &pn1);
	pp = n * (z * pn - pn1) / (z * z - 1.0);
	x[i] = z;
	x[n - 1 - i] = -z;
	const double wi = 2.0 / ((1.0 - z * z) * pp * pp);
	w[i] = wi;
	w[n - 1 - i] = wi;
	if((n & 1) && i == n / 2)
		x[i] = 0.0;
}

// normalised m = 0 Legendre table P~_l(x_i), l < LP, in both layouts
__global__ void k_plm0_table(int nt, const double *x, int LP, double *P, double *PT)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= nt)
		return;
	const double xi = x[i];
	double p0 = sqrt(1.0 / (4.0 * M_PI));
	double p1 = xi * sqrt(3.0) * p0;
	for(int l = 0; l < LP; l++) {
		double p;
		if(l == 0)
			p = p0;
		else if(l == 1)
			p = p1;
		else {
			const double a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0)) / l;
			const double b = sqrt((2.0 * l + 1.0) / (2.0 * l - 3.0)) * (l - 1.0) / l;
			p = a * xi * p1 - b * p0;
			p0 = p1;
			p1 = p;
		}
		P[(size_t) i * LP + l] = p;
		PT[(size_t) l * nt + i] = p;
	}
}

// polar projection of the sinc delay taps (projection.c:99-131): for a phase
// centre at r z-hat the mesh samples do not depend on phi, so the m = 0 bin
// of the reference's phi transform is nphi times the ring value and the tap
// is 2 pi sum_i w_i sinc(pi(-k - r x_i / dt)) P~_l(x_i).
__global__ void k_taps(double r, double dt, int n_el, int A, int nt, const double *x, const double *w, const double *P, int LP, double *taps)
{
	extern __shared__ double s_f[];
	const int t = blockIdx.x;
	const int k = t - (n_el - 1) / 2;
	for(int i = threadIdx.x; i < nt; i += blockDim.x) {
		const double pi_x = M_PI * (0 - k - r * x[i] / dt);
		const double s = (pi_x == 0.0) ? 1.0 : sin(pi_x) / pi_x;
		s_f[i] = 2.0 * M_PI * w[i] * s;
	}
	__syncthreads();
	for(int l = threadIdx.x; l < A; l += blockDim.x) {
		double acc = 0.0;
		for(int i = 0; i < nt; i++)
			acc += s_f[i] * P[(size_t) i * LP + l];
		taps[(size_t) t * A + l] = acc;
	}
}

// zero-padded DFT of the taps along the tap axis (correlator.c:446-451):
// Ahat[f][l] = sum_t taps[t][l] exp(-2 pi i f t / n), twiddles indexed
// exactly by (f t) mod n.
__global__ void k_tap_dft(int n, int n_el, int A, const double *taps, double2 *Ahat)
{
	extern __shared__ double2 s_tw[];
	const int f = blockIdx.x;
	const int n_tap = n_el < n ? n_el : n;
	for(int t = threadIdx.x; t < n_tap; t += blockDim.x) {
		const long long idx = ((long long) f * t) % n;
		double s, c;
		sincospi(-2.0 * (double) idx / n, &s, &c);
		s_tw[t] = make_double2(c, s);
	}
	__syncthreads();
	for(int l = threadIdx.x; l < A; l += blockDim.x) {
		double2 acc = make_double2(0, 0);
		for(int t = 0; t < n_tap; t++) {
			const double v = taps[(size_t) t * A + l];
			acc.x += v * s_tw[t].x;
			acc.y += v * s_tw[t].y;
		}
		Ahat[(size_t) f * A + l] = acc;
	}
}

// per-bin delay product conj(A_f) B_f truncated to l < Ld, stored at bin
// (n - f) mod n with one 1/n applied (correlator.c:482-492).  The product is
// the Gauss-Legendre quadrature of the reference's pixel-domain product
// (exact: the integrand has degree 2 a_l_max + l_max < 2 nt).  The b-side
// taps are the a-side ones mirrored in cos(theta), B_l = (-1)^l A_l, so
// sum_l B_l P~_l(x_i) = Q_f(x_{nt-1-i}) with Q_f(x) = sum_l A_l P~_l(x).
__global__ void k_delay_product(int n, int A, int nt, const double2 *Ahat, const double *PT, const double *P, int LP, const double *w, int Ld, double2 *D)
{
	extern __shared__ double2 s_mem[];
	double2 *s_a = s_mem;          // A
	double2 *s_q = s_a + A;        // nt
	double2 *s_h = s_q + nt;       // nt
	const int f = blockIdx.x;
	for(int l = threadIdx.x; l < A; l += blockDim.x)
		s_a[l] = Ahat[(size_t) f * A + l];
	__syncthreads();
	for(int i = threadIdx.x; i < nt; i += blockDim.x) {
		double2 q = make_double2(0, 0);
		for(int l = 0; l < A; l++) {
			const double p = PT[(size_t) l * nt + i];
			q.x += s_a[l].x * p;
			q.y += s_a[l].y * p;
		}
		s_q[i] = q;
	}
	__syncthreads();
	const double scale = 2.0 * M_PI / n;
	for(int i = threadIdx.x; i < nt; i += blockDim.x) {
		const double2 u = s_q[i];
		const double2 v = s_q[nt - 1 - i];
		// conj(u) * v
		const double2 h = make_double2(u.x * v.x + u.y * v.y, u.x * v.y - u.y * v.x);
		s_h[i] = make_double2(scale * w[i] * h.x, scale * w[i] * h.y);
	}
	__syncthreads();
	const size_t row = (size_t) ((n - f) % n) * Ld;
	for(int l = threadIdx.x; l < Ld; l += blockDim.x) {
		double2 acc = make_double2(0, 0);
		for(int i = 0; i < nt; i++) {
			const double p = P[(size_t) i * LP + l];
			acc.x += s_h[i].x * p;
			acc.y += s_h[i].y * p;
		}
		D[row + l] = acc;
	}
}

int build_delay_table(double d_len, double delta_t, int n, unsigned l_max, double *D_host, double **dev_out)
{
	if(ensure_device())
		return -1;
	if(!(d_len > 0) || !(delta_t > 0) || n <= 0) {
		set_error("build_delay_table: bad arguments (d=%g dt=%g n=%d)", d_len, delta_t, n);
		return -1;
	}
	const double r = d_len / 2;
	const int a_l = proj_l_max(r, delta_t);
	const int n_el = n_elements(r, delta_t);
	unsigned p_l = power_l_max_naive(d_len, delta_t);
	if(p_l > 2u * a_l)
		p_l = 2 * a_l;
	if(l_max > p_l) {
		set_error("build_delay_table: l_max %u above the baseline's power l_max %u", l_max, p_l);
		return -1;
	}
	const int A = a_l + 1;
	const int nt = 2 * A;
	const int Ld = l_max + 1;
	const int LP = A > Ld ? A : Ld;
	const size_t smem_dp = (size_t) (A + 2 * nt) * sizeof(double2);
	if(smem_dp > 200 * 1024 || (size_t) nt * sizeof(double) > 200 * 1024) {
		set_error("build_delay_table: baseline too long for this sample rate (a_l_max %d)", a_l);
		return -1;
	}
	DBuf x(nt * sizeof(double)), w(nt * sizeof(double));
	DBuf P((size_t) nt * LP * sizeof(double)), PT((size_t) nt * LP * sizeof(double));
	DBuf taps((size_t) n_el * A * sizeof(double));
	DBuf Ahat((size_t) n * A * sizeof(double2));
	double2 *D = (double2 *) dmalloc((size_t) n * Ld * sizeof(double2));
	if(!x.p || !w.p || !P.p || !PT.p || !taps.p || !Ahat.p || !D) {
		dfree(D);
		return -1;
	}
	cudaStream_t s = S();
	k_gl_nodes<<<(nt / 2 + 127) / 128, 128, 0, s>>>(nt, x.as<double>(), w.as<double>());
	k_plm0_table<<<(nt + 127) / 128, 128, 0, s>>>(nt, x.as<double>(), LP, P.as<double>(), PT.as<double>());
	k_taps<<<n_el, 256, nt * sizeof(double), s>>>(r, delta_t, n_el, A, nt, x.as<double>(), w.as<double>(), P.as<double>(), LP, taps.as<double>());
	const int n_tap = n_el < n ? n_el : n;
	k_tap_dft<<<n, 256, n_tap * sizeof(double2), s>>>(n, n_el, A, taps.as<double>(), Ahat.as<double2>());
	if(smem_dp > 48 * 1024)
		cudaFuncSetAttribute(k_delay_product, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_dp);
	k_delay_product<<<n, 256, smem_dp, s>>>(n, A, nt, Ahat.as<double2>(), PT.as<double>(), P.as<double>(), LP, w.as<double>(), Ld, D);
	cudaError_t e = cudaGetLastError();
	if(e != cudaSuccess) {
		set_error("build_delay_table: launch failed: %s", cudaGetErrorString(e));
		dfree(D);
		return -1;
	}
	if(D_host && d2h(D_host, D, (size_t) n * Ld * sizeof(double2))) {
		dfree(D);
		return -1;
	}
	if(stream_sync()) {
		dfree(D);
		return -1;
	}
	if(dev_out)
		*dev_out = (double *) D;
	else
		dfree(D);
	return 0;
}

// ------------------------------------------------------------------------
// Wigner-D rotation plan (sh_series_rotation.c:279-422)
// ------------------------------------------------------------------------
size_t rot_offset(unsigned l)
{
	// sum_{k=1}^{l-1} (2k+1)^2 = (4 l^3 - l - 3) / 3 for l >= 1
	if(l <= 1)
		return 0;
	const size_t L = l;
	return (4 * L * L * L - L - 3) / 3;
}

// One block per plan.  The l = 1 matrix (equations 5.3-5.5 of Choi et al.)
// is built from R; level l is then computed from level l - 1 and level 1,
// one element per thread, with a block barrier between levels.
constexpr int ROT_THREADS = 512;

__global__ void __launch_bounds__(ROT_THREADS) k_rotation_plan(int l_max, const double *R_all, double2 *D_all, size_t plan_stride)
{
	__shared__ double2 d1[9];
	const double *R = R_all + 9 * blockIdx.x;
	double2 *Dall = D_all + plan_stride * blockIdx.x;
	if(threadIdx.x == 0) {
		wig_d1(R, d1);
		for(int k = 0; k < 9; k++)
			Dall[k] = d1[k];
	}
	__syncthreads();
	auto D1 = [&](int m, int mp) { return d1[(mp + 1) * 3 + (m + 1)]; };
	for(int l = 2; l <= l_max; l++) {
		const double2 *Dp = Dall + wig_offset(l - 1);
		double2 *D = Dall + wig_offset(l);
		const int w = 2 * l + 1;
		const int lp = l - 1;
		for(int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
			const int m = idx % w - l;
			const int mp = idx / w - l;
			double2 v = make_double2(0, 0);
			if(mp > -l && mp < l) {
				// (6.1), (6.4), (6.5)
				if(abs(m) != l) {
					const double2 t = cmul(D1(0, 0), WDEL(Dp, lp, m, mp));
					const double c = wig_a(l, m, mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
				if(m > -l + 1) {
					const double2 t = cmul(D1(1, 0), WDEL(Dp, lp, m - 1, mp));
					const double c = wig_b(l, m, mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
				if(-m > -l + 1) {
					const double2 t = cmul(D1(-1, 0), WDEL(Dp, lp, m + 1, mp));
					const double c = wig_b(l, -m, mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
			} else if(mp == -l) {
				// (6.9), (6.12), (6.13)
				if(abs(m) != l) {
					const double2 t = cmul(D1(0, -1), WDEL(Dp, lp, m, mp + 1));
					const double c = wig_c(l, m, -mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
				if(m > -l + 1) {
					const double2 t = cmul(D1(1, -1), WDEL(Dp, lp, m - 1, mp + 1));
					const double c = wig_d(l, m, -mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
				if(-m > -l + 1) {
					const double2 t = cmul(D1(-1, -1), WDEL(Dp, lp, m + 1, mp + 1));
					const double c = wig_d(l, -m, -mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
			} else {
				// mp == l: (6.14), (6.12), (6.13)
				if(abs(m) != l) {
					const double2 t = cmul(D1(0, 1), WDEL(Dp, lp, m, mp - 1));
					const double c = wig_c(l, m, mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
				if(m > -l + 1) {
					const double2 t = cmul(D1(1, 1), WDEL(Dp, lp, m - 1, mp - 1));
					const double c = wig_d(l, m, mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
				if(-m > -l + 1) {
					const double2 t = cmul(D1(-1, 1), WDEL(Dp, lp, m + 1, mp - 1));
					const double c = wig_d(l, -m, mp);
					v.x += c * t.x;
					v.y += c * t.y;
				}
			}
			D[idx] = v;
		}
		__syncthreads();
	}
}

int build_rotation_plan(unsigned l_max, const double *R, double *D_host)
{
	if(l_max == 0)
		return 0;
	if(ensure_device())
		return -1;
	const size_t len = rot_offset(l_max + 1);
	DBuf dR(9 * sizeof(double));
	DBuf dD(len * sizeof(double2));
	if(!dR.p || !dD.p)
		return -1;
	if(h2d(dR.p, R, 9 * sizeof(double)))
		return -1;
	k_rotation_plan<<<1, ROT_THREADS, 0, S()>>>((int) l_max, dR.as<double>(), dD.as<double2>(), len);
	CK(cudaGetLastError());
	if(d2h(D_host, dD.p, len * sizeof(double2)))
		return -1;
	return stream_sync();
}

// ------------------------------------------------------------------------
// rotation of one series (sh_series_rotation.c:546-589)
// ------------------------------------------------------------------------
// grid over m' + l_max, threads over l >= |m'|.  Polar input: c'_{l m'} =
// D^l_{0 m'} c_l.  Otherwise c'_{l m'} = sum_m D^l_{m m'} c_{l m}.
__device__ __forceinline__ size_t d_lmoffset(int L, int l, int m)
{
	const long long LL = L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return (size_t) (mo + l - abs(m));
}

__global__ void k_rotate(int L, int polar, const double2 *Dall, const double2 *in, double2 *out)
{
	const int mp = (int) blockIdx.x - L;
	for(int l = abs(mp) + threadIdx.x; l <= L; l += blockDim.x) {
		double2 c;
		if(l == 0)
			c = in[0];
		else {
			const double2 *D = Dall + wig_offset(l);
			if(polar)
				c = cmul(WDEL(D, l, 0, mp), in[l]);
			else {
				c = make_double2(0, 0);
				for(int m = -l; m <= l; m++) {
					const double2 t = cmul(WDEL(D, l, m, mp), in[d_lmoffset(L, l, m)]);
					c.x += t.x;
					c.y += t.y;
				}
			}
		}
		out[d_lmoffset(L, l, mp)] = c;
	}
}

struct RotMirror {
	uint64_t gen = 0;
	unsigned l_max = 0;
	double2 *D = nullptr;
};
static std::mutex g_rot_mu;
static std::unordered_map<const void *, RotMirror> g_rot_cache;

void forget_rot_mirror(const void *key)
{
	std::lock_guard<std::mutex> lk(g_rot_mu);
	auto it = g_rot_cache.find(key);
	if(it != g_rot_cache.end()) {
		dscratch_free(it->second.D);
		g_rot_cache.erase(it);
	}
}

int rotate_series(unsigned l_max, int polar, const double *series, const double *Dflat, const void *cache_key, uint64_t gen, double *result)
{
	if(ensure_device())
		return -1;
	const size_t len = rot_offset(l_max + 1);
	double2 *dD = nullptr;
	{
		std::lock_guard<std::mutex> lk(g_rot_mu);
		RotMirror &m = g_rot_cache[cache_key];
		if(!m.D || m.gen != gen || m.l_max != l_max) {
			dscratch_free(m.D);
			m.D = (double2 *) dscratch((len ? len : 1) * sizeof(double2));
			if(!m.D)
				return -1;
			if(len && h2d(m.D, Dflat, len * sizeof(double2)))
				return -1;
			m.gen = gen;
			m.l_max = l_max;
		}
		dD = m.D;
	}
	const size_t in_len = polar ? l_max + 1 : (size_t) (l_max + 1) * (l_max + 1);
	const size_t out_len = (size_t) (l_max + 1) * (l_max + 1);
	DBuf din(in_len * sizeof(double2)), dout(out_len * sizeof(double2));
	if(!din.p || !dout.p)
		return -1;
	if(h2d(din.p, series, in_len * sizeof(double2)))
		return -1;
	k_rotate<<<2 * l_max + 1, 64, 0, S()>>>((int) l_max, polar, dD, din.as<double2>(), dout.as<double2>());
	CK(cudaGetLastError());
	if(d2h(result, dout.p, out_len * sizeof(double2)))
		return -1;
	return stream_sync();
}

// ------------------------------------------------------------------------
// FP64 frequency-domain integration (correlator.c:681-711, 993-1010)
// ------------------------------------------------------------------------
namespace {
// a typed view of a piece of the arena
struct TdSpan {
	void *p;
	template <class T_> T_ *as() const { return (T_ *) p; }
};

// grow-only device arena, per device, and grow-only pinned host staging
// buffers (one upload, one download per call) of the drop-in integrators:
// calls after the first allocate nothing while their sizes do not grow
struct TdArena {
	std::mutex mu;
	std::unordered_map<int, std::pair<void *, size_t>> bufs;
	void *hup = nullptr, *hdown = nullptr;
	size_t hup_n = 0, hdown_n = 0;
	static void *pinned(void **p, size_t *have, size_t need)
	{
		if(*have < need || !*p) {
			if(*p)
				cudaFreeHost(*p);
			*p = nullptr;
			*have = 0;
			if(cudaMallocHost(p, need ? need : 16) != cudaSuccess) {
				*p = nullptr;
				set_error("cannot allocate %zu bytes of pinned host memory", need);
				return nullptr;
			}
			*have = need;
		}
		return *p;
	}
	void *get(size_t need)
	{
		int dev = 0;
		cudaGetDevice(&dev);
		auto &b = bufs[dev];
		if(b.second < need || !b.first) {
			dfree(b.first);
			b.first = dmalloc(need);
			b.second = b.first ? need : 0;
		}
		return b.first;
	}
};
TdArena g_td_arena;
TdArena g_fd_arena;
}  // namespace

struct DevJob {
	const double2 *a, *b;   // spectra
	const double2 *D;       // n x stride delay table
	const double2 *rot;     // polar: rows D^l_{0 m'} at offset l^2; else full flat plan
	double2 *X;             // cross spectrum out (n)
	double2 *P;             // sum_k X D (stride), zeroed before the launch
	int n, stride, l_max, polar;
	double weight;
};

constexpr int XS_CHUNK = 64;

// cross-spectrum X[k] = b[k] conj(a[k]) and P[j] += sum_k X[k] D[k][j]
// (sh_series_array.c:437-456) over a chunk of XD_ROWS bins of one baseline
// per block: the block forms the chunk's X once in shared memory; warp w
// takes bins w, w + XD_WARPS, ... with its lanes over 32 consecutive j (rows
// of D read coalesced), the warps' partial sums meet in shared memory and
// one FP64 atomic per j and block leaves
constexpr int XD_ROWS = 64, XD_WARPS = 8;

__global__ void __launch_bounds__(32 * XD_WARPS) k_xdot(const DevJob *jobs)
{
	const DevJob J = jobs[blockIdx.y];
	const int k0 = blockIdx.x * XD_ROWS;
	if(k0 >= J.n)
		return;
	__shared__ double2 s_x[XD_ROWS];
	__shared__ double2 s_red[XD_WARPS][32];
	const int kc = min(XD_ROWS, J.n - k0);
	for(int k = threadIdx.x; k < kc; k += blockDim.x) {
		const double2 v = cmulc(J.b[k0 + k], J.a[k0 + k]);
		s_x[k] = v;
		if(J.X)
			J.X[k0 + k] = v;
	}
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for(int j0 = 0; j0 < J.stride; j0 += 32) {
		const int j = j0 + lane;
		double2 acc = make_double2(0, 0);
		if(j < J.stride) {
			const double2 *d = J.D + (size_t) k0 * J.stride + j;
#pragma unroll 4
			for(int k = warp; k < kc; k += XD_WARPS) {
				const double2 t = cmul(d[(size_t) k * J.stride], s_x[k]);
				acc.x += t.x;
				acc.y += t.y;
			}
		}
		s_red[warp][lane] = acc;
		__syncthreads();
		if(warp == 0 && j < J.stride) {
			double2 v = s_red[0][lane];
			for(int w = 1; w < XD_WARPS; w++) {
				v.x += s_red[w][lane].x;
				v.y += s_red[w][lane].y;
			}
			atomicAdd(&J.P[j].x, v.x);
			atomicAdd(&J.P[j].y, v.y);
		}
		__syncthreads();
	}
}

// sky_{l m'} = sum_b weight_b / n_b * (rotated P_b)_{l m'} (grid: m' + L,
// threads over l); with pw set, block b < n_jobs also writes baseline b's
// power_1d = P_b / n_b to pw + b * pw_stride
__global__ void k_rotate_sum(const DevJob *jobs, int n_jobs, int L, double2 *sky, double2 *pw = nullptr, int pw_stride = 0)
{
	if(pw && (int) blockIdx.x < n_jobs) {
		const DevJob &J = jobs[blockIdx.x];
		for(int j = threadIdx.x; j < J.stride; j += blockDim.x) {
			const double2 p = J.P[j];
			pw[(size_t) blockIdx.x * pw_stride + j] = make_double2(p.x / J.n, p.y / J.n);
		}
	}
	const int mp = (int) blockIdx.x - L;
	if(mp > L)
		return;
	for(int l = abs(mp) + threadIdx.x; l <= L; l += blockDim.x) {
		double2 acc = make_double2(0, 0);
		for(int b = 0; b < n_jobs; b++) {
			const DevJob &J = jobs[b];
			if(l > J.l_max)
				continue;
			const double s = J.weight / J.n;
			double2 c;
			if(l == 0)
				c = J.P[0];
			else if(J.polar)
				c = cmul(J.rot[(size_t) l * l + (mp + l)], J.P[l]);
			else {
				c = make_double2(0, 0);
				const double2 *D = J.rot + wig_offset(l);
				for(int m = -l; m <= l; m++) {
					const double2 t = cmul(WDEL(D, l, m, mp), J.P[d_lmoffset(J.l_max, l, m)]);
					c.x += t.x;
					c.y += t.y;
				}
			}
			acc.x += s * c.x;
			acc.y += s * c.y;
		}
		sky[d_lmoffset(L, l, mp)] = acc;
	}
}

// device mirror of a plan: delay table and rotation data
struct PlanMirror {
	uint64_t gen = ~0ull;
	const double *D_host = nullptr;
	const double *rot_host = nullptr;
	int n = 0, stride = 0, polar = -1;
	unsigned l_max = 0;
	double2 *D = nullptr;
	double2 *rot = nullptr;
};
static std::mutex g_mir_mu;
static std::unordered_map<const void *, PlanMirror> g_mirrors;

void forget_mirror(const void *key)
{
	std::lock_guard<std::mutex> lk(g_mir_mu);
	auto it = g_mirrors.find(key);
	if(it != g_mirrors.end()) {
		dfree(it->second.D);
		dfree(it->second.rot);
		g_mirrors.erase(it);
	}
}

static int refresh_mirror(const BaselineJob &j, PlanMirror &m)
{
	if(m.D && m.gen == j.gen && m.D_host == j.D && m.rot_host == j.rot && m.n == j.n && m.stride == j.stride && m.l_max == j.l_max && m.polar == j.polar)
		return 0;
	dfree(m.D);
	dfree(m.rot);
	m.D = m.rot = nullptr;
	m.D = (double2 *) dmalloc((size_t) j.n * j.stride * sizeof(double2));
	if(!m.D)
		return -1;
	if(h2d(m.D, j.D, (size_t) j.n * j.stride * sizeof(double2)))
		return -1;
	if(j.polar) {
		// rows D^l_{0 m'} at offset l^2, l = 0 row is 1
		const size_t rl = (size_t) (j.l_max + 1) * (j.l_max + 1);
		std::vector<double> rows(2 * rl, 0.0);
		rows[0] = 1.0;
		for(unsigned l = 1; l <= j.l_max; l++) {
			const double *Dl = j.rot + 2 * rot_offset(l);
			for(int mp = -(int) l; mp <= (int) l; mp++) {
				const size_t e = (size_t) (2 * l + 1) * (mp + l) + (0 + l);
				rows[2 * ((size_t) l * l + mp + l)] = Dl[2 * e];
				rows[2 * ((size_t) l * l + mp + l) + 1] = Dl[2 * e + 1];
			}
		}
		m.rot = (double2 *) dmalloc(rl * sizeof(double2));
		if(!m.rot || h2d(m.rot, rows.data(), rl * sizeof(double2)) || stream_sync())
			return -1;
	} else {
		const size_t len = rot_offset(j.l_max + 1);
		m.rot = (double2 *) dmalloc((len ? len : 1) * sizeof(double2));
		if(!m.rot || (len && h2d(m.rot, j.rot, len * sizeof(double2))))
			return -1;
	}
	m.gen = j.gen;
	m.D_host = j.D;
	m.rot_host = j.rot;
	m.n = j.n;
	m.stride = j.stride;
	m.l_max = j.l_max;
	m.polar = j.polar;
	return 0;
}

int integrate_fd(const BaselineJob *jobs, int n_jobs, unsigned sky_l_max, double *sky)
{
	if(ensure_device())
		return -1;
	if(n_jobs <= 0) {
		set_error("integrate_fd: no baselines");
		return -1;
	}
	std::vector<DevJob> dj(n_jobs);
	// unique input spectra (the network shares detectors between baselines)
	std::vector<const double *> uniq;
	std::vector<int> uniq_n;
	auto find_or_add = [&](const double *p, int n) {
		for(size_t i = 0; i < uniq.size(); i++)
			if(uniq[i] == p && uniq_n[i] == n)
				return (int) i;
		uniq.push_back(p);
		uniq_n.push_back(n);
		return (int) uniq.size() - 1;
	};
	std::vector<int> ia(n_jobs), ib(n_jobs);
	size_t spec_total = 0, x_total = 0, p_total = 0;
	int max_n = 0, max_stride = 0;
	for(int i = 0; i < n_jobs; i++) {
		const BaselineJob &J = jobs[i];
		if(J.n <= 0 || J.stride <= 0 || J.l_max > sky_l_max) {
			set_error("integrate_fd: bad baseline job %d", i);
			return -1;
		}
		ia[i] = find_or_add(J.a, J.n);
		ib[i] = find_or_add(J.b, J.n);
		x_total += J.n;
		p_total += J.stride;
		max_n = J.n > max_n ? J.n : max_n;
		max_stride = J.stride > max_stride ? J.stride : max_stride;
	}
	for(size_t i = 0; i < uniq.size(); i++)
		spec_total += uniq_n[i];
	const size_t sky_len = (size_t) (sky_l_max + 1) * (sky_l_max + 1);
	// one grow-only device arena per device, held for the call: an upload
	// region (unique spectra, job table) filled by one copy from pinned
	// staging, a download region (sky, power_1d rows, cross spectra) read
	// back by one copy, and the partial sums P
	auto al = [](size_t b) { return (b + 255) & ~(size_t) 255; };
	const size_t up_spec = al(spec_total * sizeof(double2));
	const size_t up_bytes = up_spec + al(n_jobs * sizeof(DevJob));
	const size_t dn_sky = al(sky_len * sizeof(double2));
	const size_t dn_pw = al((size_t) n_jobs * max_stride * sizeof(double2));
	const size_t dn_bytes = dn_sky + dn_pw + x_total * sizeof(double2);
	const size_t p_bytes = p_total * sizeof(double2);
	std::lock_guard<std::mutex> lock(g_fd_arena.mu);
	char *base = (char *) g_fd_arena.get(up_bytes + al(dn_bytes) + p_bytes);
	char *hup = (char *) TdArena::pinned(&g_fd_arena.hup, &g_fd_arena.hup_n, up_bytes);
	char *hdown = (char *) TdArena::pinned(&g_fd_arena.hdown, &g_fd_arena.hdown_n, dn_bytes);
	if(!base || !hup || !hdown)
		return -1;
	double2 *spec = (double2 *) base;
	DevJob *djobs = (DevJob *) (base + up_spec);
	char *down = base + up_bytes;
	double2 *dsky = (double2 *) down;
	double2 *pw = (double2 *) (down + dn_sky);
	double2 *X = (double2 *) (down + dn_sky + dn_pw);
	double2 *P = (double2 *) (base + up_bytes + al(dn_bytes));
	std::vector<size_t> uoff(uniq.size());
	{
		size_t o = 0;
		for(size_t i = 0; i < uniq.size(); i++) {
			uoff[i] = o;
			memcpy(hup + o * sizeof(double2), uniq[i], uniq_n[i] * sizeof(double2));
			o += uniq_n[i];
		}
	}
	size_t xo = 0, po = 0;
	{
		std::lock_guard<std::mutex> lk(g_mir_mu);
		for(int i = 0; i < n_jobs; i++) {
			const BaselineJob &J = jobs[i];
			PlanMirror &m = g_mirrors[J.key];
			if(refresh_mirror(J, m))
				return -1;
			DevJob &d = dj[i];
			d.a = spec + uoff[ia[i]];
			d.b = spec + uoff[ib[i]];
			d.D = m.D;
			d.rot = m.rot;
			d.X = X + xo;
			d.P = P + po;
			d.n = J.n;
			d.stride = J.stride;
			d.l_max = (int) J.l_max;
			d.polar = J.polar;
			d.weight = J.weight;
			xo += J.n;
			po += J.stride;
		}
	}
	memcpy(hup + up_spec, dj.data(), n_jobs * sizeof(DevJob));
	CK(cudaMemcpyAsync(base, hup, up_bytes, cudaMemcpyHostToDevice, S()));
	CK(cudaMemsetAsync(P, 0, p_bytes, S()));
	dim3 g1((max_n + XD_ROWS - 1) / XD_ROWS, n_jobs);
	k_xdot<<<g1, 32 * XD_WARPS, 0, S()>>>(djobs);
	const int rgrid = (int) (2 * sky_l_max + 1) > n_jobs ? (int) (2 * sky_l_max + 1) : n_jobs;
	k_rotate_sum<<<rgrid, 64, 0, S()>>>(djobs, n_jobs, (int) sky_l_max, dsky, pw, max_stride);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(hdown, down, dn_bytes, cudaMemcpyDeviceToHost, S()));
	if(stream_sync())
		return -1;
	memcpy(sky, hdown, sky_len * sizeof(double2));
	xo = 0;
	for(int i = 0; i < n_jobs; i++) {
		const BaselineJob &J = jobs[i];
		if(J.power_1d)
			memcpy(J.power_1d, hdown + dn_sky + (size_t) i * max_stride * sizeof(double2), J.stride * sizeof(double2));
		if(J.fseries_product)
			memcpy(J.fseries_product, hdown + dn_sky + dn_pw + xo * sizeof(double2), J.n * sizeof(double2));
		xo += J.n;
	}
	return 0;
}

// ------------------------------------------------------------------------
// array contraction (sh_series_array.c:404-456)
// ------------------------------------------------------------------------
__global__ void k_array_dot(int n, int stride, const double2 *coeff, const double2 *vec, double2 *out)
{
	const int k0 = blockIdx.x * XS_CHUNK;
	const int kc = min(XS_CHUNK, n - k0);
	__shared__ double2 s_v[XS_CHUNK];
	for(int k = threadIdx.x; k < kc; k += blockDim.x)
		s_v[k] = vec[k0 + k];
	__syncthreads();
	for(int j = threadIdx.x; j < stride; j += blockDim.x) {
		double2 acc = make_double2(0, 0);
		for(int k = 0; k < kc; k++) {
			const double2 t = cmul(coeff[(size_t) (k0 + k) * stride + j], s_v[k]);
			acc.x += t.x;
			acc.y += t.y;
		}
		atomicAdd(&out[j].x, acc.x);
		atomicAdd(&out[j].y, acc.y);
	}
}

int array_dotc(int n, int stride, const double *coeff, const double *vec, int vec_is_complex, double *result)
{
	if(ensure_device())
		return -1;
	if(n <= 0) {
		memset(result, 0, stride * sizeof(double2));
		return 0;
	}
	DBuf dc((size_t) n * stride * sizeof(double2)), dv((size_t) n * sizeof(double2)), dout(stride * sizeof(double2));
	if(!dc.p || !dv.p || !dout.p)
		return -1;
	std::vector<double> v2;
	const double *vp = vec;
	if(!vec_is_complex) {
		v2.assign(2 * (size_t) n, 0.0);
		for(int k = 0; k < n; k++)
			v2[2 * k] = vec[k];
		vp = v2.data();
	}
	if(h2d(dc.p, coeff, (size_t) n * stride * sizeof(double2)) || h2d(dv.p, vp, n * sizeof(double2)) || dmemset(dout.p, 0, stride * sizeof(double2)))
		return -1;
	k_array_dot<<<(n + XS_CHUNK - 1) / XS_CHUNK, 128, 0, S()>>>(n, stride, dc.as<double2>(), dv.as<double2>(), dout.as<double2>());
	CK(cudaGetLastError());
	if(d2h(result, dout.p, stride * sizeof(double2)))
		return -1;
	return stream_sync();
}

}  // namespace sphrad

namespace sphrad {

// ------------------------------------------------------------------------
// time-domain correlator (correlator.c:325-400, 648-673)
//
// The reference loops over the n - 2 transient samples: it forms each
// sample's polar series on both sides (sh_series_array_dot of the
// projection taps with the series from that sample), multiplies them
// (sh_series_product) and adds the product, times the window, into
// power_1d.  The product is bilinear, so the window-weighted sum of
// products is the product contraction of one matrix,
//     C[l1][l2] = sum_t w[t] Sa[t][l1] Sb[t][l2],
// and power_1d[L] = sum_{l1,l2} C[l1][l2] int Y_L0 Y_l1,0 Y_l2,0, which a
// Gauss-Legendre rule in cos(theta) of (P + La + Lb) / 2 + 1 nodes
// integrates exactly (the quadrature of the pixel-domain product,
// sh_series_product.c:269-329).  Samples and C are tiled FP64 kernels;
// the per-sample product loop disappears.
// ------------------------------------------------------------------------
int projection_taps(double r, double delta_t, int n_el, int A, double *taps_host)
{
	if(!(delta_t > 0) || n_el <= 0 || A <= 0) {
		set_error("projection taps: bad sample interval %g or shape %d x %d", delta_t, n_el, A);
		return -1;
	}
	const int nt = 2 * A;
	if(ensure_device())
		return -1;
	DBuf x(nt * sizeof(double)), w(nt * sizeof(double)), P((size_t) nt * A * sizeof(double)), PT((size_t) nt * A * sizeof(double)),
		taps((size_t) n_el * A * sizeof(double));
	if(!x.p || !w.p || !P.p || !PT.p || !taps.p)
		return -1;
	cudaStream_t s = S();
	k_gl_nodes<<<(nt / 2 + 127) / 128, 128, 0, s>>>(nt, x.as<double>(), w.as<double>());
	k_plm0_table<<<(nt + 127) / 128, 128, 0, s>>>(nt, x.as<double>(), A, P.as<double>(), PT.as<double>());
	k_taps<<<n_el, 256, nt * sizeof(double), s>>>(r, delta_t, n_el, A, nt, x.as<double>(), w.as<double>(), P.as<double>(), A, taps.as<double>());
	CK(cudaGetLastError());
	if(d2h(taps_host, taps.p, (size_t) n_el * A * sizeof(double)) || stream_sync())
		return -1;
	return 0;
}

namespace {

constexpr int kTdTT = 64, kTdTL = 32, kTdTE = 32;  // samples tile: t x l, taps chunk

// S[t][l] = sum_e taps[e][l] x[t + e], t < T, l < A (sh_series_array_dot
// from each sample, sh_series_array.c:407-426).  Block: 64 samples x 32
// harmonics, 256 threads, 8 samples per thread.
// REAL: every tap is real (the polar projections of a phase centre on the
// z axis are), so only the real parts are formed; the imaginary parts are
// written as zeros
template <bool REAL>
__global__ void __launch_bounds__(256) k_td_samples(int T, int n_el, int A, const double2 *__restrict__ taps, const double *__restrict__ x, double2 *__restrict__ S)
{
	__shared__ double2 s_tap[kTdTE][kTdTL];
	__shared__ double s_x[kTdTT + kTdTE];
	const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
	const int t0 = blockIdx.x * kTdTT, l0 = blockIdx.y * kTdTL;
	double2 acc[8];
#pragma unroll
	for(int k = 0; k < 8; k++)
		acc[k] = make_double2(0.0, 0.0);
	for(int e0 = 0; e0 < n_el; e0 += kTdTE) {
		for(int i = threadIdx.x; i < kTdTE * kTdTL; i += blockDim.x) {
			const int e = e0 + i / kTdTL, l = l0 + i % kTdTL;
			s_tap[i / kTdTL][i % kTdTL] = (e < n_el && l < A) ? taps[(size_t) e * A + l] : make_double2(0.0, 0.0);
		}
		// samples with t < T and e < n_el read x below T + n_el - 1, the
		// length of the staged series; the rest of the window is zero
		for(int j = threadIdx.x; j < kTdTT + kTdTE; j += blockDim.x) {
			const long long idx = (long long) t0 + e0 + j;
			s_x[j] = idx < (long long) T + n_el - 1 ? x[idx] : 0.0;
		}
		__syncthreads();
		const int ne = n_el - e0 < kTdTE ? n_el - e0 : kTdTE;
		for(int e = 0; e < ne; e++) {
			const double2 c = s_tap[e][tx];
#pragma unroll
			for(int k = 0; k < 8; k++) {
				const double v = s_x[ty + 8 * k + e];
				acc[k].x += c.x * v;
				if(!REAL)
					acc[k].y += c.y * v;
			}
		}
		__syncthreads();
	}
	const int l = l0 + tx;
	if(l < A)
#pragma unroll
		for(int k = 0; k < 8; k++) {
			const int t = t0 + ty + 8 * k;
			if(t < T)
				S[(size_t) t * A + l] = acc[k];
		}
}

// partial C over the sample range of blockIdx.z:
// part[z][l1][l2] = sum_t w[t] Sa[t][l1] Sb[t][l2].  Block: 32 x 32
// outputs, 256 threads, 4 per thread.  REAL: the samples are real (real
// taps), so are C's entries.
template <bool REAL>
__global__ void __launch_bounds__(256) k_td_cross(int T, int t_per, int Aa, int Ab, const double *__restrict__ w, const double2 *__restrict__ Sa,
						  const double2 *__restrict__ Sb, double2 *__restrict__ part)
{
	__shared__ double2 s_a[32][33];
	__shared__ double2 s_b[32][32];
	const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
	const int l10 = blockIdx.y * 32, l20 = blockIdx.x * 32;
	const int tb = blockIdx.z * t_per, te = tb + t_per < T ? tb + t_per : T;
	double2 acc[4];
#pragma unroll
	for(int k = 0; k < 4; k++)
		acc[k] = make_double2(0.0, 0.0);
	for(int t0 = tb; t0 < te; t0 += 32) {
		for(int i = threadIdx.x; i < 32 * 32; i += blockDim.x) {
			const int tt = i / 32, j = i % 32, t = t0 + tt;
			const bool ok = t < te;
			const double wt = ok ? w[t] : 0.0;
			const double2 a = (ok && l10 + j < Aa) ? Sa[(size_t) t * Aa + l10 + j] : make_double2(0.0, 0.0);
			const double2 b = (ok && l20 + j < Ab) ? Sb[(size_t) t * Ab + l20 + j] : make_double2(0.0, 0.0);
			s_a[tt][j] = a;
			s_b[tt][j] = make_double2(wt * b.x, wt * b.y);
		}
		__syncthreads();
#pragma unroll 4
		for(int tt = 0; tt < 32; tt++) {
			const double2 b = s_b[tt][tx];
#pragma unroll
			for(int k = 0; k < 4; k++) {
				const double2 a = s_a[tt][ty + 8 * k];
				if(REAL)
					acc[k].x += a.x * b.x;
				else {
					acc[k].x += a.x * b.x - a.y * b.y;
					acc[k].y += a.x * b.y + a.y * b.x;
				}
			}
		}
		__syncthreads();
	}
	const int l2 = l20 + tx;
	if(l2 < Ab)
#pragma unroll
		for(int k = 0; k < 4; k++) {
			const int l1 = l10 + ty + 8 * k;
			if(l1 < Aa)
				part[((size_t) blockIdx.z * Aa + l1) * Ab + l2] = acc[k];
		}
}

// fixed-order sum of a 256-thread block's values (thread 0 gets it)
__device__ double2 td_block_sum(double2 v)
{
	__shared__ double2 s_red[256];
	s_red[threadIdx.x] = v;
	__syncthreads();
	for(int s = blockDim.x / 2; s > 0; s >>= 1) {
		if(threadIdx.x < s) {
			s_red[threadIdx.x].x += s_red[threadIdx.x + s].x;
			s_red[threadIdx.x].y += s_red[threadIdx.x + s].y;
		}
		__syncthreads();
	}
	return s_red[0];
}

// C = sum over the partials: one warp per element, lanes over the
// partials, a fixed shuffle tree (the same order on every run)
__global__ void k_td_reduce(int nz, size_t len, const double2 *__restrict__ part, double2 *__restrict__ C)
{
	const size_t w = (blockIdx.x * (size_t) blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if(w >= len)
		return;  // whole warps leave together
	double2 acc = make_double2(0.0, 0.0);
	for(int z = lane; z < nz; z += 32) {
		const double2 v = part[(size_t) z * len + w];
		acc.x += v.x;
		acc.y += v.y;
	}
#pragma unroll
	for(int o = 16; o > 0; o >>= 1) {
		acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
		acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
	}
	if(lane == 0)
		C[w] = acc;
}

// q[i] = sum_{l1,l2} P~_l1(x_i) C[l1][l2] P~_l2(x_i), one 256-thread block
// per node: lanes over l2, the 8 warps over l1
__global__ void __launch_bounds__(256) k_td_node(int nq, int LP, int Aa, int Ab, const double *__restrict__ P, const double2 *__restrict__ C,
						 double2 *__restrict__ q)
{
	const int i = blockIdx.x, lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
	const double *Pi = P + (size_t) i * LP;
	double2 acc = make_double2(0.0, 0.0);
	for(int l2 = lane; l2 < Ab; l2 += 32) {
		double2 g = make_double2(0.0, 0.0);
		for(int l1 = grp; l1 < Aa; l1 += 8) {
			const double2 c = C[(size_t) l1 * Ab + l2];
			g.x += Pi[l1] * c.x;
			g.y += Pi[l1] * c.y;
		}
		acc.x += g.x * Pi[l2];
		acc.y += g.y * Pi[l2];
	}
	const double2 t = td_block_sum(acc);
	if(threadIdx.x == 0)
		q[i] = t;
}

// power[L] = 2 pi sum_i w_i q_i P~_L(x_i), one 256-thread block per L <= Lp
// (PT: the degree-major table, PT[L][i])
__global__ void __launch_bounds__(256) k_td_power(int nq, const double *__restrict__ wq, const double *__restrict__ PT, const double2 *__restrict__ q,
						  double2 *__restrict__ power)
{
	const int L = blockIdx.x;
	const double *PL = PT + (size_t) L * nq;
	double2 acc = make_double2(0.0, 0.0);
	for(int i = threadIdx.x; i < nq; i += blockDim.x) {
		const double f = wq[i] * PL[i];
		acc.x += f * q[i].x;
		acc.y += f * q[i].y;
	}
	const double2 t = td_block_sum(acc);
	if(threadIdx.x == 0)
		power[L] = make_double2(2.0 * M_PI * t.x, 2.0 * M_PI * t.y);
}


}  // namespace

// shapes of one baseline's time-domain pass
struct TdShape {
	int T, n_ela, n_elb, Aa, Ab, nq, LP, nz, t_per;
	unsigned Lp;
	size_t clen;
	bool real;  // every tap real
};

// true when every imaginary part of the complex [n][A] taps is zero
static bool taps_real(const double *taps, int n, int A)
{
	for(size_t i = 0; i < (size_t) n * A; i++)
		if(taps[2 * i + 1] != 0.0)
			return false;
	return true;
}

static TdShape td_shape(int T, int n_ela, int n_elb, int Aa, int Ab, unsigned Lp, bool real)
{
	TdShape h;
	h.real = real;
	h.T = T;
	h.n_ela = n_ela;
	h.n_elb = n_elb;
	h.Aa = Aa;
	h.Ab = Ab;
	h.Lp = Lp;
	h.nq = ((int) Lp + (Aa - 1) + (Ab - 1)) / 2 + 1;
	h.LP = std::max(std::max(Aa, Ab), (int) Lp + 1);
	h.clen = (size_t) Aa * Ab;
	// split the sample sum so that about four blocks per SM run
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const int tiles = ((Aa + 31) / 32) * ((Ab + 31) / 32);
	int nz = (4 * sms + tiles - 1) / tiles;
	nz = std::max(1, std::min(nz, (T + 63) / 64));
	h.t_per = ((T + nz - 1) / nz + 31) / 32 * 32;
	h.nz = std::max(1, (T + h.t_per - 1) / h.t_per);
	return h;
}

// device scratch of one pass: taps a, taps b, window, S_a, S_b, partials,
// C, nodes, weights, P, PT, q, power
constexpr int kTdBufs = 13;

static void td_sizes(const TdShape &h, size_t *sz)
{
	const size_t T = (size_t) h.T;
	const size_t v[kTdBufs] = {(size_t) h.n_ela * h.Aa * 16, (size_t) h.n_elb * h.Ab * 16, T * 8, T * h.Aa * 16, T * h.Ab * 16, (size_t) h.nz * h.clen * 16,
				   h.clen * 16, (size_t) h.nq * 8, (size_t) h.nq * 8, (size_t) h.nq * h.LP * 8, (size_t) h.nq * h.LP * 8, (size_t) h.nq * 16,
				   ((size_t) h.Lp + 1) * 16};
	for(int i = 0; i < kTdBufs; i++)
		sz[i] = (v[i] + 255) / 256 * 256;
}

// the kernels of one pass; xa, xb: device series; b[]: the buffers of
// td_sizes; power_1d lands in b[12]
static int td_launch(const TdShape &h, const double *xa, const double *xb, char *const *b, cudaStream_t s)
{
	const int T = h.T, Aa = h.Aa, Ab = h.Ab, nq = h.nq, LP = h.LP;
	if(T == 0) {
		CK(cudaMemsetAsync(b[12], 0, ((size_t) h.Lp + 1) * 16, s));
		return 0;
	}
	const double2 *ta = (const double2 *) b[0], *tb = (const double2 *) b[1];
	const double *w = (const double *) b[2];
	double2 *Sa = (double2 *) b[3], *Sb = (double2 *) b[4], *part = (double2 *) b[5], *C = (double2 *) b[6], *q = (double2 *) b[11], *pw = (double2 *) b[12];
	double *x = (double *) b[7], *wq = (double *) b[8], *P = (double *) b[9], *PT = (double *) b[10];
	const dim3 ga((T + kTdTT - 1) / kTdTT, (Aa + kTdTL - 1) / kTdTL), gb((T + kTdTT - 1) / kTdTT, (Ab + kTdTL - 1) / kTdTL),
		gc((Ab + 31) / 32, (Aa + 31) / 32, h.nz);
	if(h.real) {
		k_td_samples<true><<<ga, 256, 0, s>>>(T, h.n_ela, Aa, ta, xa, Sa);
		k_td_samples<true><<<gb, 256, 0, s>>>(T, h.n_elb, Ab, tb, xb, Sb);
		k_td_cross<true><<<gc, 256, 0, s>>>(T, h.t_per, Aa, Ab, w, Sa, Sb, part);
	} else {
		k_td_samples<false><<<ga, 256, 0, s>>>(T, h.n_ela, Aa, ta, xa, Sa);
		k_td_samples<false><<<gb, 256, 0, s>>>(T, h.n_elb, Ab, tb, xb, Sb);
		k_td_cross<false><<<gc, 256, 0, s>>>(T, h.t_per, Aa, Ab, w, Sa, Sb, part);
	}
	k_td_reduce<<<(int) ((h.clen * 32 + 255) / 256), 256, 0, s>>>(h.nz, h.clen, part, C);
	k_gl_nodes<<<(nq / 2 + 1 + 127) / 128, 128, 0, s>>>(nq, x, wq);
	k_plm0_table<<<(nq + 127) / 128, 128, 0, s>>>(nq, x, LP, P, PT);
	k_td_node<<<nq, 256, 0, s>>>(nq, LP, Aa, Ab, P, C, q);
	k_td_power<<<(int) h.Lp + 1, 256, 0, s>>>(nq, wq, PT, q, pw);
	CK(cudaGetLastError());
	return 0;
}

static bool td_valid(int T, int n_ela, int n_elb, int Aa, int Ab, long long n_x)
{
	return T >= 0 && n_ela > 0 && n_elb > 0 && Aa > 0 && Ab > 0 && (long long) T + n_ela - 1 <= n_x && (long long) T + n_elb - 1 <= n_x;
}

int td_power_1d(int T, int n_ela, int n_elb, int Aa, int Ab, const double *taps_a, const double *taps_b, const double *xa, const double *xb, long long n_x,
		const double *w, unsigned Lp, double *power_host)
{
	if(!td_valid(T, n_ela, n_elb, Aa, Ab, n_x)) {
		set_error("time-domain correlator: %d samples of %lld with %d- and %d-tap projections", T, n_x, n_ela, n_elb);
		return -1;
	}
	if(T == 0) {
		memset(power_host, 0, ((size_t) Lp + 1) * 2 * sizeof(double));
		return 0;
	}
	if(ensure_device())
		return -1;
	const TdShape h = td_shape(T, n_ela, n_elb, Aa, Ab, Lp, taps_real(taps_a, n_ela, Aa) && taps_real(taps_b, n_elb, Ab));
	size_t sz[kTdBufs];
	td_sizes(h, sz);
	const size_t xa_b = ((size_t) (T + n_ela - 1) * 8 + 255) / 256 * 256, xb_b = ((size_t) (T + n_elb - 1) * 8 + 255) / 256 * 256;
	size_t total = xa_b + xb_b;
	for(int i = 0; i < kTdBufs; i++)
		total += sz[i];
	// one grow-only device arena per device, held for the whole call
	std::lock_guard<std::mutex> lock(g_td_arena.mu);
	char *base = (char *) g_td_arena.get(total);
	if(!base)
		return -1;
	char *dxa = base, *dxb = base + xa_b, *b[kTdBufs];
	size_t o = xa_b + xb_b;
	for(int i = 0; i < kTdBufs; i++) {
		b[i] = base + o;
		o += sz[i];
	}
	if(h2d(b[0], taps_a, (size_t) n_ela * Aa * 16) || h2d(b[1], taps_b, (size_t) n_elb * Ab * 16) || h2d(dxa, xa, (size_t) (T + n_ela - 1) * 8) ||
	   h2d(dxb, xb, (size_t) (T + n_elb - 1) * 8) || h2d(b[2], w, (size_t) T * 8))
		return -1;
	if(td_launch(h, (const double *) dxa, (const double *) dxb, b, S()))
		return -1;
	if(d2h(power_host, b[12], ((size_t) Lp + 1) * 16) || stream_sync())
		return -1;
	return 0;
}

int td_network(const TdBaseline *bl, int nb, int n_det, long long n, const double *const *series, double weight, unsigned sky_L, double *sky_host)
{
	if(nb <= 0 || n_det <= 0 || n <= 0) {
		set_error("time-domain network: %d baselines, %d detectors, %lld samples", nb, n_det, n);
		return -1;
	}
	for(int k = 0; k < nb; k++) {
		const TdBaseline &B = bl[k];
		if(!td_valid(B.T, B.n_ela, B.n_elb, B.Aa, B.Ab, n) || B.det_a < 0 || B.det_a >= n_det || B.det_b < 0 || B.det_b >= n_det || B.Lp > sky_L ||
		   B.Lp > (unsigned) (B.Aa - 1 + B.Ab - 1)) {
			set_error("time-domain network: baseline %d does not fit (%d samples of %lld, l_max %u of %u)", k, B.T, n, B.Lp, sky_L);
			return -1;
		}
	}
	if(ensure_device())
		return -1;
	// device arena: an upload region (series, jobs, then per baseline taps a,
	// taps b, window, rotation rows) filled by one copy from pinned staging,
	// a download region (sky, then per baseline power_1d) read back by one
	// copy, and the scratch of every baseline's pass
	std::vector<TdShape> sh(nb);
	std::vector<size_t> sz((size_t) nb * kTdBufs), rot_b(nb), up_off(nb), pw_off(nb), sc_off(nb);
	const size_t ser_b = ((size_t) n_det * n * 8 + 255) / 256 * 256, sky_len = ((size_t) sky_L + 1) * (sky_L + 1);
	const size_t sky_b = (sky_len * 16 + 255) / 256 * 256, job_b = ((size_t) nb * sizeof(DevJob) + 255) / 256 * 256;
	size_t up = ser_b + job_b, down = sky_b, scratch = 0;
	for(int k = 0; k < nb; k++) {
		sh[k] = td_shape(bl[k].T, bl[k].n_ela, bl[k].n_elb, bl[k].Aa, bl[k].Ab, bl[k].Lp,
				 taps_real(bl[k].taps_a, bl[k].n_ela, bl[k].Aa) && taps_real(bl[k].taps_b, bl[k].n_elb, bl[k].Ab));
		const size_t *z = &sz[(size_t) k * kTdBufs];
		td_sizes(sh[k], &sz[(size_t) k * kTdBufs]);
		rot_b[k] = (((size_t) bl[k].Lp + 1) * (bl[k].Lp + 1) * 16 + 255) / 256 * 256;
		up_off[k] = up;
		up += z[0] + z[1] + z[2] + rot_b[k];
		pw_off[k] = down;
		down += z[12];
		sc_off[k] = scratch;
		for(int i = 3; i < 12; i++)
			scratch += z[i];
	}
	std::lock_guard<std::mutex> lock(g_td_arena.mu);
	char *base = (char *) g_td_arena.get(up + down + scratch);
	char *hup = (char *) TdArena::pinned(&g_td_arena.hup, &g_td_arena.hup_n, up);
	char *hdown = (char *) TdArena::pinned(&g_td_arena.hdown, &g_td_arena.hdown_n, down);
	if(!base || !hup || !hdown)
		return -1;
	char *dser = base, *djobs = base + ser_b, *dsky = base + up;
	for(int d = 0; d < n_det; d++)
		memcpy(hup + (size_t) d * n * 8, series[d], (size_t) n * 8);
	std::vector<DevJob> dj(nb);
	std::vector<std::array<char *, kTdBufs>> bufs(nb);
	for(int k = 0; k < nb; k++) {
		const TdBaseline &B = bl[k];
		const size_t *z = &sz[(size_t) k * kTdBufs];
		char **b = bufs[k].data();
		b[0] = base + up_off[k];
		b[1] = b[0] + z[0];
		b[2] = b[1] + z[1];
		char *drot = b[2] + z[2];
		size_t o = up + down + sc_off[k];
		for(int i = 3; i < 12; i++) {
			b[i] = base + o;
			o += z[i];
		}
		b[12] = base + up + pw_off[k];
		char *h = hup + up_off[k];
		memcpy(h, B.taps_a, (size_t) B.n_ela * B.Aa * 16);
		memcpy(h + z[0], B.taps_b, (size_t) B.n_elb * B.Ab * 16);
		if(B.T > 0)
			memcpy(h + z[0] + z[1], B.window, (size_t) B.T * 8);
		memcpy(h + z[0] + z[1] + z[2], B.rot_rows, ((size_t) B.Lp + 1) * (B.Lp + 1) * 16);
		// the rotation and network sum (correlator.c:665-670, 976-981) as
		// the FD integrator's: power_1d is already normalised (n = 1)
		DevJob &J = dj[k];
		memset(&J, 0, sizeof(J));
		J.rot = (const double2 *) drot;
		J.P = (double2 *) b[12];
		J.n = 1;
		J.stride = (int) B.Lp + 1;
		J.l_max = (int) B.Lp;
		J.polar = 1;
		J.weight = weight;
	}
	memcpy(hup + ser_b, dj.data(), (size_t) nb * sizeof(DevJob));
	cudaStream_t s = S();
	CK(cudaMemcpyAsync(base, hup, up, cudaMemcpyHostToDevice, s));
	for(int k = 0; k < nb; k++) {
		const TdBaseline &B = bl[k];
		if(td_launch(sh[k], (const double *) (dser + (size_t) B.det_a * n * 8), (const double *) (dser + (size_t) B.det_b * n * 8), bufs[k].data(), s))
			return -1;
	}
	k_rotate_sum<<<2 * sky_L + 1, 64, 0, s>>>((const DevJob *) djobs, nb, (int) sky_L, (double2 *) dsky);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(hdown, dsky, down, cudaMemcpyDeviceToHost, s));
	if(stream_sync())
		return -1;
	memcpy(sky_host, hdown, sky_len * 16);
	for(int k = 0; k < nb; k++)
		if(bl[k].power_host)
			memcpy(bl[k].power_host, hdown + pw_off[k], ((size_t) bl[k].Lp + 1) * 16);
	return 0;
}

}  // namespace sphrad
