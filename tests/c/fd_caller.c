/*
 * A C caller of the drop-in frequency-domain path, written the way a
 * program of the reference project calls it (src/bin/sphradiometer_demo.c:
 * instruments, network baselines, network plan, then
 * correlator_network_integrate_power_fd once per segment), compiled against
 * the repository's include/sphradiometer headers and linked with
 * libsphradiometer_b200.so.
 *
 *   fd_caller in.bin out.bin
 *
 * in.bin (little-endian): int32 n_det, int32 n, int32 l_max, int32 n_seg,
 * float64 delta_t, float64 positions[n_det][3] (light-seconds), then per
 * segment and detector n complex128 bins (the full spectrum).  out.bin:
 * per segment the (l_max + 1)^2 complex128 coefficients of the sky.
 * Exit status 0 on success.
 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>

#include <sphradiometer/correlator.h>
#include <sphradiometer/instrument.h>
#include <sphradiometer/sh_series.h>

static int read_all(FILE *f, void *p, size_t bytes)
{
	return fread(p, 1, bytes, f) == bytes ? 0 : -1;
}

int main(int argc, char *argv[])
{
	if(argc != 3) {
		fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
		return 2;
	}
	FILE *in = fopen(argv[1], "rb");
	FILE *out = fopen(argv[2], "wb");
	if(!in || !out)
		return 2;
	int hdr[4];
	double delta_t;
	if(read_all(in, hdr, sizeof(hdr)) || read_all(in, &delta_t, sizeof(delta_t)))
		return 3;
	const int n_det = hdr[0], n = hdr[1], l_max = hdr[2], n_seg = hdr[3];
	double *pos = malloc(sizeof(double) * 3 * n_det);
	if(!pos || read_all(in, pos, sizeof(double) * 3 * n_det))
		return 3;

	struct instrument_array *instruments = instrument_array_new(0);
	for(int d = 0; d < n_det; d++)
		if(!instrument_array_append(instruments, instrument_new(pos[3 * d], pos[3 * d + 1], pos[3 * d + 2], NULL)))
			return 4;
	struct correlator_network_baselines *baselines = correlator_network_baselines_new(instruments);
	struct correlator_network_plan_fd *plan = baselines ? correlator_network_plan_fd_new_l(baselines, n, delta_t, (unsigned) l_max) : NULL;
	struct sh_series *sky = sh_series_new((unsigned) l_max, 0);
	double complex **fseries = malloc(sizeof(*fseries) * n_det);
	if(!plan || !sky || !fseries)
		return 4;
	for(int d = 0; d < n_det; d++)
		if(!(fseries[d] = malloc(sizeof(double complex) * n)))
			return 4;

	for(int s = 0; s < n_seg; s++) {
		for(int d = 0; d < n_det; d++)
			if(read_all(in, fseries[d], sizeof(double complex) * n))
				return 3;
		if(!correlator_network_integrate_power_fd(sky, fseries, plan))
			return 5;
		const size_t len = (size_t) (l_max + 1) * (l_max + 1);
		if(fwrite(sky->coeff, sizeof(double complex), len, out) != len)
			return 6;
	}

	for(int d = 0; d < n_det; d++)
		free(fseries[d]);
	free(fseries);
	sh_series_free(sky);
	correlator_network_plan_fd_free(plan);
	correlator_network_baselines_free(baselines);
	instrument_array_free(instruments);
	free(pos);
	fclose(in);
	return fclose(out) ? 6 : 0;
}
