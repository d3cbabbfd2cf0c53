/*
 * dqmc_batch: runs many sim files as chains of one GPU run.  Files with
 * identical parameters share kernel launches.  Options as dqmc_1 (-t, -l, -b);
 * exit status 0 if every file completed, 1 if any stopped early, -1 (255) if
 * any failed.  Takes the place of many dqmc_stack processes
 * (src/main_stack.c) for files that fit one GPU.
 */
#include <argp.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>

#include "dqmc_b200.h"

static struct argp_option options[] = {
	{0, 't', "TIME", 0, "Max allowed wall time in integer seconds", 0},
	{"log", 'l', "LOGFILE", 0, "Redirect stdout to LOGFILE", 0},
	{"benchmark", 'b', 0, 0, "Don't save sim_data to disk", 0},
	{0}};

struct arguments {
	int time;
	char *log_file;
	bool bench;
	int n;
	char **files;
};

static error_t parse_opt(int key, char *arg, struct argp_state *state)
{
	struct arguments *a = state->input;
	switch (key) {
	case 't': a->time = atoi(arg); break;
	case 'l': a->log_file = arg; break;
	case 'b': a->bench = true; break;
	case ARGP_KEY_ARG:
		a->files = realloc(a->files, sizeof(char *) * (a->n + 1));
		a->files[a->n++] = arg;
		break;
	case ARGP_KEY_END:
		if (state->arg_num < 1) argp_usage(state);
		break;
	default: return ARGP_ERR_UNKNOWN;
	}
	return 0;
}

static struct argp argp = {options, parse_opt, "sim_file.h5 [sim_file.h5 ...]",
                           "DQMC sweeps of many sim files on one B200 GPU", 0, 0, 0};

int main(int argc, char **argv)
{
	struct arguments a = {0, NULL, false, 0, NULL};
	argp_parse(&argp, argc, argv, 0, 0, &a);
	int *status = calloc(a.n, sizeof(int));
	const int rc = dqmc_wrapper_batch(a.n, (const char *const *)a.files, a.log_file, (int64_t)a.time * 1000000000LL,
	                                  a.bench, status);
	for (int i = 0; i < a.n; i++) printf("%s %d\n", a.files[i], status[i]);
	free(status);
	free(a.files);
	return rc;
}
