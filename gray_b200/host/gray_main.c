/*
 * `gray` -- command-line driver of the GRay2 job, the equivalent of
 * `lux gray opt=value ...` (README.md:16-21): construct the job, hand every
 * argument to conf(), then init() and exec().
 */
#include <stdio.h>

#include "gray_job.h"

int
main(int argc, char **argv)
{
	gray_lux_job *job = gray_job_mkmod(NULL);
	int st;
	if(!job) {
		fprintf(stderr, "gray: out of memory\n");
		return 1;
	}
	for(int i = 1; i < argc; ++i) {
		st = job->conf(job, argv[i]);
		if(st) {
			fprintf(stderr, "gray: %s option \"%s\"\n",
			        st == GRAY_JOB_UNKNOWN ? "unknown" : "invalid", argv[i]);
			gray_job_rmmod(job);
			return 2;
		}
	}
	if((st = job->init(job)) || (st = job->exec(job))) {
		fprintf(stderr, "gray: %s\n", gray_strerror(st));
		gray_job_rmmod(job);
		return 1;
	}
	gray_job_rmmod(job);
	return 0;
}
