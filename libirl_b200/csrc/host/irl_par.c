/* irl_par.c -- a loop split over the host's cores, for the element-wise
   passes of the set-up (layout reorders, clamps, scalings, fills).  Each
   element is computed exactly as in a serial loop, so the results do not
   depend on the number of threads.  Loops that accumulate (libirl's float
   sums) stay serial. */
#include <pthread.h>
#include <unistd.h>

#include "irl_host.h"

#define IRL_PAR_MAX 16

typedef struct {
	irl_range_fn fn;
	void *ctx;
	size_t lo, hi;
} par_job;

static void *par_run(void *a)
{
	par_job *j = (par_job *)a;
	j->fn(j->lo, j->hi, j->ctx);
	return NULL;
}

void irl_parallel_for(size_t n, size_t grain, irl_range_fn fn, void *ctx)
{
	long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
	size_t t = ncpu > 0 ? (size_t)ncpu : 1, i;
	pthread_t th[IRL_PAR_MAX];
	par_job job[IRL_PAR_MAX];
	int started[IRL_PAR_MAX];
	if (t > IRL_PAR_MAX)
		t = IRL_PAR_MAX;
	if (grain < 1)
		grain = 1;
	if (t > n / grain)
		t = n / grain;
	if (t <= 1) {
		fn(0, n, ctx);
		return;
	}
	for (i = 0; i < t; ++i) {
		job[i].fn = fn;
		job[i].ctx = ctx;
		job[i].lo = n * i / t;
		job[i].hi = n * (i + 1) / t;
	}
	for (i = 1; i < t; ++i)
		started[i] = pthread_create(&th[i], NULL, par_run, &job[i]) == 0;
	par_run(&job[0]);
	for (i = 1; i < t; ++i) {
		if (started[i])
			pthread_join(th[i], NULL);
		else
			par_run(&job[i]); /* no thread could be started: run the chunk here */
	}
}
