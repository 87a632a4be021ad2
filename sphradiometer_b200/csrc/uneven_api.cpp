// uneven_api.cpp -- uneven batches: segments of different DFT lengths,
// output l_max and baseline subsets of one detector network integrated in
// one call (declared in sphradiometer_b200.h; no reference counterpart --
// the reference integrates one segment of one network per call,
// correlator.c:993-1010, and its callers pad segments to a length ladder,
// inspiral_sky_map.c's preprocessing).
//
// Plan: segments are bucketed by DFT length (the delay tables depend on
// n).  Each segment's baselines are covered by sub-networks of at most
// three detectors (the tcgen05 contraction's limit), greedily; every
// (bucket, sub-network) pair with segments is a job: a batched plan of that
// sub-network at the bucket's n and the plan's l_max, the job's segment
// list and per-segment baseline factors (n_sub_baselines / B_s for the
// segment's baselines assigned to the job, 0 otherwise, so each sky is the
// mean over its own B_s baselines, correlator.c:1004).  A call zeroes the
// packed outputs and runs every job: the contraction reads the job's
// segments where they lie in the caller's packed spectra (the FP32 / FP64
// precisions gather them first) and the epilogue adds each segment's sky
// into its packed output, truncated to the segment's own l_max (FP64
// atomics: a segment covered by two jobs gets the same sum in either
// order).  Each job runs its own contraction and epilogue, the jobs spread
// over a few streams (longest first, each to the least loaded stream); for
// the tcgen05 precisions (by default; per-job launches on request) all
// jobs' contractions run in one persistent launch (batch_contract_multi)
// and the jobs' epilogues are forked over the streams.  The whole sequence can be captured once into a CUDA graph and
// replayed.
#include <sphradiometer_b200.h>
#include <sphradiometer/correlator.h>
#include <sphradiometer/instrument.h>

#include <cuda_runtime_api.h>

#include <algorithm>
#include <map>
#include <vector>

#include "abi_common.h"

using namespace sphrad;

namespace {

struct Job {
	int bucket = 0;
	std::vector<int> det;        // detectors of the sub-network (increasing)
	std::vector<int> gbl;        // global baseline ids of its baselines, in its plan's order
	sphrad_batch_plan *bp = nullptr;
	int S = 0, Ku = 0;
	long long ld = 0;
	std::vector<int> seg;        // host copies
	std::vector<float> w;        // [S][nb_sub]
	int *d_seg = nullptr;
	float *d_w = nullptr;
	long long *d_rowoff = nullptr;  // [S] the segments' rows in the packed spectra
	long long *d_outrow = nullptr;  // [S] their skies in the packed outputs
	unsigned *d_segL = nullptr;     // [S] their l_max
	bool indexed = false;           // tcgen05 precision: spectra read in place
	int split = 0;               // tuned split (0 = heuristic)
	int slot = 0;                // stream and scratch slot
};

constexpr int kSlots = 4;        // streams the jobs are spread over

}  // namespace

struct sphrad_uneven_plan {
	int n_det = 0;
	double dt = 0;
	std::vector<double> pos;
	std::vector<int> bucket_n;
	unsigned L = 0;
	int precision = 0;
	int nbl = 0;                                     // baselines of the full network
	std::vector<std::pair<int, int>> bl;             // global baseline id -> (i, j), i > j
	// sub-networks: detector lists; per (bucket, sub) a batched plan
	std::vector<std::vector<int>> subs;
	std::map<std::pair<int, int>, sphrad_batch_plan *> plans;
	std::vector<void *> net_objs;                    // instruments, baselines, network plans to free
	// segments
	int n_seg = 0;
	std::vector<unsigned> segL;
	std::vector<long long> in_off, out_off;
	long long in_total = 0, out_total = 0;
	long long *d_in_off = nullptr, *d_out_off = nullptr;
	unsigned *d_segL = nullptr;
	std::vector<Job> jobs;
	// job buffers: gathered spectra (FP32 / FP64 jobs and the autotuner)
	// and split-K scratch per slot (the jobs of a slot run in sequence);
	// the autotuner's skies of one job
	void *F = nullptr, *sky = nullptr, *ws = nullptr;
	size_t F_bytes = 0, sky_bytes = 0, ws_bytes = 0;
	int n_slots = 1;
	cudaStream_t side[kSlots] = {};
	cudaEvent_t ev[kSlots + 1] = {};
	int fixed_split = 0;
	// persistent launch (tcgen05 precisions, the default): every job's
	// contraction in one launch, each job with its own zeroed workspace at
	// ws_off
	int persistent = 1;
	void *ws_multi = nullptr;
	std::vector<size_t> ws_off;
	// graph
	int use_graph = 1;
	cudaStream_t cap = nullptr;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	const void *g_in = nullptr;
	void *g_out = nullptr;
	int g_split = -1;
	int kernels = 0;
};

static void drop_graph(sphrad_uneven_plan *p)
{
	if(p->exec)
		cudaGraphExecDestroy(p->exec);
	if(p->graph)
		cudaGraphDestroy(p->graph);
	p->exec = nullptr;
	p->graph = nullptr;
	p->g_in = nullptr;
	p->g_out = nullptr;
}

static void drop_jobs(sphrad_uneven_plan *p)
{
	for(Job &j : p->jobs) {
		dfree(j.d_seg);
		dfree(j.d_w);
		dfree(j.d_rowoff);
		dfree(j.d_outrow);
		dfree(j.d_segL);
	}
	p->jobs.clear();
	dfree(p->d_in_off);
	dfree(p->d_out_off);
	dfree(p->d_segL);
	p->d_in_off = p->d_out_off = nullptr;
	p->d_segL = nullptr;
	dfree(p->F);
	dfree(p->sky);
	dfree(p->ws);
	dfree(p->ws_multi);
	p->F = p->sky = p->ws = p->ws_multi = nullptr;
	p->ws_off.clear();
	p->F_bytes = p->sky_bytes = p->ws_bytes = 0;
	drop_graph(p);
}

extern "C" void sphrad_uneven_plan_free(sphrad_uneven_plan *p)
{
	if(!p)
		return;
	drop_jobs(p);
	for(auto &kv : p->plans)
		sphrad_batch_plan_free(kv.second);
	// network objects: plan, baselines, instruments (in creation order of
	// triples: [inst_array, baselines, plan] per (bucket, sub))
	for(size_t i = 0; i + 2 < p->net_objs.size(); i += 3) {
		correlator_network_plan_fd_free((struct correlator_network_plan_fd *) p->net_objs[i + 2]);
		correlator_network_baselines_free((struct correlator_network_baselines *) p->net_objs[i + 1]);
		instrument_array_free((struct instrument_array *) p->net_objs[i]);
	}
	if(p->cap)
		cudaStreamDestroy(p->cap);
	for(int k = 0; k < kSlots; k++)
		if(p->side[k])
			cudaStreamDestroy(p->side[k]);
	for(int k = 0; k <= kSlots; k++)
		if(p->ev[k])
			cudaEventDestroy(p->ev[k]);
	delete p;
}

extern "C" sphrad_uneven_plan *sphrad_uneven_plan_new(const double *positions, int n_det, double delta_t, const int *bucket_n, int n_buckets, unsigned l_max,
						     int precision)
{
	if(n_det < 2 || n_det > 8 || n_buckets < 1 || !positions || !bucket_n) {
		set_error("sphrad_uneven_plan_new: %d detectors, %d buckets", n_det, n_buckets);
		return NULL;
	}
	if(ensure_device())
		return NULL;
	sphrad_uneven_plan *p = new sphrad_uneven_plan;
	p->n_det = n_det;
	p->dt = delta_t;
	p->pos.assign(positions, positions + 3 * n_det);
	p->bucket_n.assign(bucket_n, bucket_n + n_buckets);
	p->L = l_max;
	p->precision = precision;
	for(int i = 1; i < n_det; i++)
		for(int j = 0; j < i; j++)
			p->bl.push_back({i, j});
	p->nbl = (int) p->bl.size();
	// sub-networks of min(3, n_det) detectors
	if(n_det <= 3) {
		std::vector<int> all;
		for(int d = 0; d < n_det; d++)
			all.push_back(d);
		p->subs.push_back(all);
	} else {
		for(int a = 0; a < n_det; a++)
			for(int b = a + 1; b < n_det; b++)
				for(int c = b + 1; c < n_det; c++)
					p->subs.push_back({a, b, c});
	}
	bool ok = cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking) == cudaSuccess;
	for(int k = 1; ok && k < kSlots; k++)
		ok = cudaStreamCreateWithFlags(&p->side[k], cudaStreamNonBlocking) == cudaSuccess;
	for(int k = 0; ok && k <= kSlots; k++)
		ok = cudaEventCreateWithFlags(&p->ev[k], cudaEventDisableTiming) == cudaSuccess;
	if(!ok) {
		set_error("sphrad_uneven_plan_new: stream creation failed");
		sphrad_uneven_plan_free(p);
		return NULL;
	}
	return p;
}

// global baseline id of (i, j), i > j, in the reference's order
static int gid(int i, int j) { return i * (i - 1) / 2 + j; }

static sphrad_batch_plan *plan_for(sphrad_uneven_plan *p, int bucket, int sub)
{
	auto key = std::make_pair(bucket, sub);
	auto it = p->plans.find(key);
	if(it != p->plans.end())
		return it->second;
	const std::vector<int> &dets = p->subs[sub];
	struct instrument_array *ia = instrument_array_new(0);
	if(!ia)
		return NULL;
	for(int d : dets) {
		struct instrument *ins = instrument_new(p->pos[3 * d], p->pos[3 * d + 1], p->pos[3 * d + 2], NULL);
		if(!ins || !instrument_array_append(ia, ins)) {
			instrument_array_free(ia);
			return NULL;
		}
	}
	struct correlator_network_baselines *nb = correlator_network_baselines_new(ia);
	struct correlator_network_plan_fd *np = nb ? correlator_network_plan_fd_new_l(nb, p->bucket_n[bucket], p->dt, p->L) : NULL;
	sphrad_batch_plan *bp = np ? sphrad_batch_plan_new(np, p->precision) : NULL;
	p->net_objs.push_back(ia);
	p->net_objs.push_back(nb);
	p->net_objs.push_back(np);
	if(!bp)
		return NULL;
	p->plans[key] = bp;
	return bp;
}

extern "C" int sphrad_uneven_set_segments(sphrad_uneven_plan *p, int n_seg, const int *bucket, const unsigned *mask, const unsigned *l_max)
{
	drop_jobs(p);
	if(n_seg < 0) {
		set_error("sphrad_uneven_set_segments: %d segments", n_seg);
		return -1;
	}
	p->n_seg = n_seg;
	p->segL.assign(l_max, l_max + n_seg);
	p->in_off.resize(n_seg);
	p->out_off.resize(n_seg);
	long long io = 0, oo = 0;
	const int nb_sub = p->n_det <= 3 ? p->nbl : 3;
	// job index per (bucket, sub)
	std::map<std::pair<int, int>, int> job_of;
	for(int s = 0; s < n_seg; s++) {
		const int b = bucket[s];
		if(b < 0 || b >= (int) p->bucket_n.size() || l_max[s] > p->L) {
			set_error("sphrad_uneven_set_segments: segment %d has bucket %d, l_max %u", s, b, l_max[s]);
			return -1;
		}
		const unsigned full = p->nbl >= 32 ? 0xFFFFFFFFu : ((1u << p->nbl) - 1);
		const unsigned m = mask[s] & full;
		const int Bs = __builtin_popcount(m);
		if(Bs == 0) {
			set_error("sphrad_uneven_set_segments: segment %d has no baseline", s);
			return -1;
		}
		const int Ku = p->bucket_n[b] / 2 + 1;
		p->in_off[s] = io;
		io += (long long) p->n_det * Ku;
		p->out_off[s] = oo;
		oo += (long long) (l_max[s] + 1) * (l_max[s] + 1);
		// greedy cover of the segment's baselines by sub-networks
		unsigned left = m;
		while(left) {
			int best = -1, best_cnt = 0;
			for(int t = 0; t < (int) p->subs.size(); t++) {
				int cnt = 0;
				const std::vector<int> &d = p->subs[t];
				for(size_t x = 0; x < d.size(); x++)
					for(size_t y = 0; y < x; y++)
						cnt += (left >> gid(d[x], d[y])) & 1;
				if(cnt > best_cnt) {
					best_cnt = cnt;
					best = t;
				}
			}
			auto key = std::make_pair(b, best);
			auto it = job_of.find(key);
			int ji;
			if(it == job_of.end()) {
				ji = (int) p->jobs.size();
				job_of[key] = ji;
				Job j;
				j.bucket = b;
				j.det = p->subs[best];
				// the sub-network plan's baseline order: (1,0), (2,0), (2,1)
				for(size_t x = 1; x < j.det.size(); x++)
					for(size_t y = 0; y < x; y++)
						j.gbl.push_back(gid(j.det[x], j.det[y]));
				j.Ku = Ku;
				j.ld = Ku;
				p->jobs.push_back(j);
			} else
				ji = it->second;
			Job &j = p->jobs[ji];
			j.seg.push_back(s);
			for(int g : j.gbl) {
				const bool take = (left >> g) & 1;
				j.w.push_back(take ? (float) nb_sub / (float) Bs : 0.f);
				if(take)
					left &= ~(1u << g);
			}
		}
	}
	p->in_total = io;
	p->out_total = oo;
	// device tables and buffers
	size_t Fb = 0, skb = 0, wsb = 0;
	const size_t nq = (size_t) (p->L + 1) * (p->L + 1);
	for(Job &j : p->jobs) {
		skb = std::max(skb, (size_t) j.seg.size() * nq * 16);
		j.S = (int) j.seg.size();
		j.bp = plan_for(p, j.bucket, (int) (std::find(p->subs.begin(), p->subs.end(), j.det) - p->subs.begin()));
		if(!j.bp)
			return -1;
		j.indexed = batch_is_tc(j.bp) != 0;
		std::vector<long long> ro(j.S), oro(j.S);
		std::vector<unsigned> sl(j.S);
		for(int i = 0; i < j.S; i++) {
			ro[i] = p->in_off[j.seg[i]];
			oro[i] = p->out_off[j.seg[i]];
			sl[i] = p->segL[j.seg[i]];
		}
		j.d_seg = (int *) dmalloc(j.S * sizeof(int));
		j.d_w = (float *) dmalloc(j.w.size() * sizeof(float));
		j.d_rowoff = (long long *) dmalloc(j.S * sizeof(long long));
		j.d_outrow = (long long *) dmalloc(j.S * sizeof(long long));
		j.d_segL = (unsigned *) dmalloc(j.S * sizeof(unsigned));
		if(!j.d_seg || !j.d_w || !j.d_rowoff || !j.d_outrow || !j.d_segL || h2d(j.d_seg, j.seg.data(), j.S * sizeof(int)) ||
		   h2d(j.d_w, j.w.data(), j.w.size() * sizeof(float)) || h2d(j.d_rowoff, ro.data(), j.S * sizeof(long long)) ||
		   h2d(j.d_outrow, oro.data(), j.S * sizeof(long long)) || h2d(j.d_segL, sl.data(), j.S * sizeof(unsigned)))
			return -1;
		Fb = std::max(Fb, (size_t) (j.det.size() * j.S * j.ld * 16));
		wsb = std::max(wsb, sphrad_batch_workspace_size(j.bp, j.S));
	}
	// slots: longest job first to the least loaded slot (cost ~ S n_sub Ku)
	p->n_slots = std::min(kSlots, std::max(1, (int) p->jobs.size()));
	{
		std::vector<int> order(p->jobs.size());
		for(size_t i = 0; i < order.size(); i++)
			order[i] = (int) i;
		auto cost = [&](int i) { return (double) p->jobs[i].S * p->jobs[i].det.size() * p->jobs[i].Ku; };
		std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
		std::vector<double> load(p->n_slots, 0.0);
		for(int i : order) {
			const int k = (int) (std::min_element(load.begin(), load.end()) - load.begin());
			p->jobs[i].slot = k;
			load[k] += cost(i);
		}
	}
	Fb = (Fb + 255) / 256 * 256;
	wsb = (wsb + 255) / 256 * 256;
	p->d_in_off = (long long *) dmalloc((n_seg > 0 ? n_seg : 1) * sizeof(long long));
	p->d_out_off = (long long *) dmalloc((n_seg > 0 ? n_seg : 1) * sizeof(long long));
	p->d_segL = (unsigned *) dmalloc((n_seg > 0 ? n_seg : 1) * sizeof(unsigned));
	p->F = dmalloc(Fb * p->n_slots);
	p->sky = dmalloc(skb ? skb : 16);
	p->ws = dmalloc(wsb * p->n_slots);
	p->F_bytes = Fb;
	p->sky_bytes = skb;
	p->ws_bytes = wsb;
	if(!p->d_in_off || !p->d_out_off || !p->d_segL || !p->F || !p->sky || !p->ws)
		return -1;
	if(n_seg > 0 && (h2d(p->d_in_off, p->in_off.data(), n_seg * sizeof(long long)) || h2d(p->d_out_off, p->out_off.data(), n_seg * sizeof(long long)) ||
			 h2d(p->d_segL, p->segL.data(), n_seg * sizeof(unsigned))))
		return -1;
	if(dmemset(p->ws, 0, wsb * p->n_slots) || stream_sync())
		return -1;
	// the persistent launch's workspaces: one per job, side by side
	bool all_indexed = !p->jobs.empty();
	for(const Job &j : p->jobs)
		all_indexed = all_indexed && j.indexed;
	if(all_indexed) {
		size_t tot = 0;
		for(const Job &j : p->jobs) {
			p->ws_off.push_back(tot);
			tot += (batch_job_ws_bytes(batch_impl(j.bp), j.S) + 255) / 256 * 256;
		}
		p->ws_multi = dmalloc(tot ? tot : 256);
		if(!p->ws_multi || dmemset(p->ws_multi, 0, tot ? tot : 256) || stream_sync())
			return -1;
	}
	return 0;
}

extern "C" int sphrad_uneven_layout(const sphrad_uneven_plan *p, long long *in_offset, long long *out_offset, long long *in_total, long long *out_total)
{
	if(in_offset)
		std::copy(p->in_off.begin(), p->in_off.end(), in_offset);
	if(out_offset)
		std::copy(p->out_off.begin(), p->out_off.end(), out_offset);
	if(in_total)
		*in_total = p->in_total;
	if(out_total)
		*out_total = p->out_total;
	return p->n_seg;
}

extern "C" int sphrad_uneven_jobs(const sphrad_uneven_plan *p) { return (int) p->jobs.size(); }

static int split_of(const sphrad_uneven_plan *p, const Job &j)
{
	if(p->fixed_split > 0)
		return p->fixed_split;
	return j.split;
}

// spectra, scratch and skies of job j
static void *job_F(sphrad_uneven_plan *p, const Job &j) { return (char *) p->F + (size_t) j.slot * p->F_bytes; }
static void *job_ws(sphrad_uneven_plan *p, const Job &j) { return (char *) p->ws + (size_t) j.slot * p->ws_bytes; }
static void *job_sky(sphrad_uneven_plan *p, const Job &) { return p->sky; }

// the outputs zeroed, every job's contraction in one persistent launch on
// st, then the jobs' epilogues forked over the slots' streams and joined
// back
static int run_persistent(sphrad_uneven_plan *p, const void *in, void *out, cudaStream_t st)
{
	cudaStream_t ss[kSlots];
	ss[0] = st;
	for(int s = 1; s < p->n_slots; s++)
		ss[s] = p->side[s];
	if(cudaMemsetAsync(out, 0, (size_t) p->out_total * 16, st) != cudaSuccess) {
		set_error("uneven: output zeroing failed");
		return -1;
	}
	std::vector<MultiJob> mj(p->jobs.size());
	for(size_t i = 0; i < p->jobs.size(); i++) {
		const Job &j = p->jobs[i];
		MultiJob &m = mj[i];
		m.plan = batch_impl(j.bp);
		m.S = j.S;
		m.ix.row_off = j.d_rowoff;
		for(size_t d = 0; d < j.det.size() && d < 3; d++)
			m.ix.det_off[d] = (long long) j.det[d] * j.Ku;
		m.ix.out_row = j.d_outrow;
		m.ix.seg_L = j.d_segL;
		m.ix.accumulate = 1;
		m.segw = j.d_w;
		m.ws = (char *) p->ws_multi + p->ws_off[i];
	}
	const int nl = batch_contract_multi(mj.data(), (int) mj.size(), in, st, 0);
	if(nl < 0)
		return -1;
	if(cudaEventRecord(p->ev[0], st) != cudaSuccess) {
		set_error("uneven: event record failed");
		return -1;
	}
	for(int s = 1; s < p->n_slots; s++)
		if(cudaStreamWaitEvent(ss[s], p->ev[0], 0) != cudaSuccess) {
			set_error("uneven: stream fork failed");
			return -1;
		}
	for(size_t i = 0; i < mj.size(); i++)
		if(batch_epilogue_job(mj[i], out, ss[i % p->n_slots]))
			return -1;
	for(int s = 1; s < p->n_slots; s++)
		if(cudaEventRecord(p->ev[s], ss[s]) != cudaSuccess || cudaStreamWaitEvent(st, p->ev[s], 0) != cudaSuccess) {
			set_error("uneven: stream join failed");
			return -1;
		}
	p->kernels = nl + (int) mj.size();
	return 0;
}

// the jobs forked over the slots' streams from st, each its own
// contraction and epilogue, joined back
static int run_jobs(sphrad_uneven_plan *p, const void *in, void *out, cudaStream_t st)
{
	if(p->persistent && p->ws_multi)
		return run_persistent(p, in, out, st);
	int k = 0;
	cudaStream_t ss[kSlots];
	ss[0] = st;
	for(int s = 1; s < p->n_slots; s++)
		ss[s] = p->side[s];
	// the jobs add into the packed outputs
	if(cudaMemsetAsync(out, 0, (size_t) p->out_total * 16, st) != cudaSuccess || cudaEventRecord(p->ev[0], st) != cudaSuccess) {
		set_error("uneven: output zeroing or event record failed");
		return -1;
	}
	for(int s = 1; s < p->n_slots; s++)
		if(cudaStreamWaitEvent(ss[s], p->ev[0], 0) != cudaSuccess) {
			set_error("uneven: stream fork failed");
			return -1;
		}
	for(Job &j : p->jobs) {
		cudaStream_t js = ss[j.slot];
		BatchIdx ix;
		ix.out_row = j.d_outrow;
		ix.seg_L = j.d_segL;
		ix.accumulate = 1;
		const void *F = in;
		if(j.indexed) {
			ix.row_off = j.d_rowoff;
			for(size_t d = 0; d < j.det.size() && d < 3; d++)
				ix.det_off[d] = (long long) j.det[d] * j.Ku;
		} else {
			if(uneven_gather(j.S, (int) j.det.size(), j.Ku, j.ld, j.d_seg, p->d_in_off, j.det.data(), in, job_F(p, j), js))
				return -1;
			F = job_F(p, j);
			k++;
		}
		if(batch_integrate_packed(j.bp, F, j.S, j.ld, &ix, out, job_ws(p, j), p->ws_bytes, js, split_of(p, j), j.d_w))
			return -1;
		k += sphrad_batch_kernels_per_call(j.bp);
	}
	for(int s = 1; s < p->n_slots; s++)
		if(cudaEventRecord(p->ev[s], ss[s]) != cudaSuccess || cudaStreamWaitEvent(st, p->ev[s], 0) != cudaSuccess) {
			set_error("uneven: stream join failed");
			return -1;
		}
	p->kernels = k;
	return 0;
}

extern "C" int sphrad_uneven_set_split(sphrad_uneven_plan *p, int split)
{
	p->fixed_split = split > 0 ? split : 0;
	drop_graph(p);
	return 0;
}

extern "C" int sphrad_uneven_set_persistent(sphrad_uneven_plan *p, int on)
{
	p->persistent = on ? 1 : 0;
	drop_graph(p);
	return 0;
}

extern "C" int sphrad_uneven_persistent(const sphrad_uneven_plan *p) { return p->persistent && p->ws_multi ? 1 : 0; }

extern "C" int sphrad_uneven_use_graph(sphrad_uneven_plan *p, int on)
{
	p->use_graph = on ? 1 : 0;
	drop_graph(p);
	return 0;
}

extern "C" int sphrad_uneven_autotune(sphrad_uneven_plan *p, const void *in, void *out, void *stream)
{
	cudaStream_t st = stream ? (cudaStream_t) stream : cudaStreamLegacy;
	(void) out;
	for(Job &j : p->jobs) {
		if(uneven_gather(j.S, (int) j.det.size(), j.Ku, j.ld, j.d_seg, p->d_in_off, j.det.data(), in, job_F(p, j), st))
			return -1;
		// the job's plan keeps the tuned work split for j.S
		if(sphrad_batch_autotune(j.bp, job_F(p, j), j.S, j.ld, job_sky(p, j), job_ws(p, j), p->ws_bytes, st) < 0)
			return -1;
		j.split = 0;
	}
	drop_graph(p);
	return 0;
}

extern "C" int sphrad_uneven_integrate(sphrad_uneven_plan *p, const void *in, void *out, void *stream)
{
	cudaStream_t st = stream ? (cudaStream_t) stream : cudaStreamLegacy;
	if(p->n_seg == 0)
		return 0;
	if(!p->use_graph)
		return run_jobs(p, in, out, st);
	if(!p->exec || p->g_in != in || p->g_out != out) {
		drop_graph(p);
		// capture on the plan's own stream, ordered after the caller's work
		cudaEvent_t ev;
		if(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(ev, st) != cudaSuccess ||
		   cudaStreamWaitEvent(p->cap, ev, 0) != cudaSuccess) {
			set_error("uneven: cannot order the capture stream");
			return -1;
		}
		cudaEventDestroy(ev);
		if(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
			set_error("uneven: stream capture failed to start");
			return -1;
		}
		const int rc = run_jobs(p, in, out, p->cap);
		cudaGraph_t g = nullptr;
		const cudaError_t ec = cudaStreamEndCapture(p->cap, &g);
		if(rc || ec != cudaSuccess || !g) {
			if(g)
				cudaGraphDestroy(g);
			if(!rc)
				set_error("uneven: stream capture failed (%s)", cudaGetErrorString(ec));
			return -1;
		}
		p->graph = g;
		if(cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) {
			set_error("uneven: graph instantiation failed");
			drop_graph(p);
			return -1;
		}
		p->g_in = in;
		p->g_out = out;
	}
	if(cudaGraphLaunch(p->exec, st) != cudaSuccess) {
		set_error("uneven: graph launch failed");
		return -1;
	}
	return 0;
}

extern "C" int sphrad_uneven_kernels_per_call(const sphrad_uneven_plan *p) { return p->kernels; }
