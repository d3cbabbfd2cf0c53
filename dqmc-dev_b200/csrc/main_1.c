/*
 * dqmc_1: single sim file CLI.  Same options and exit status as the
 * reference's src/main_1.c:20-114 (-t max wall seconds, -n dry run,
 * -l log file, -b benchmark mode; exit status = dqmc_wrapper's return).
 * -t is converted to the nanoseconds dqmc_wrapper takes, so the limit is
 * the number of seconds the option's help text promises (the reference's
 * main_1.c:103 passes the number unconverted, as nanoseconds).
 */
#include <argp.h>
#include <stdbool.h>
#include <stdlib.h>

#include "dqmc_b200.h"

static struct argp_option options[] = {
	{0, 't', "TIME", 0, "Max allowed wall time in integer seconds", 0},
	{"dry-run", 'n', 0, 0, "Report memory requirement only", 0},
	{"log", 'l', "LOGFILE", 0, "Redirect stdout to LOGFILE", 0},
	{"benchmark", 'b', 0, 0, "Don't save sim_data to disk", 0},
	{0}};

struct arguments {
	int time;
	char *log_file;
	bool dry_run, bench;
	char *file;
};

static error_t parse_opt(int key, char *arg, struct argp_state *state)
{
	struct arguments *a = state->input;
	switch (key) {
	case 't': a->time = atoi(arg); break;
	case 'l': a->log_file = arg; break;
	case 'n': a->dry_run = true; break;
	case 'b': a->bench = true; break;
	case ARGP_KEY_ARG:
		if (state->arg_num >= 1) argp_usage(state);
		a->file = arg;
		break;
	case ARGP_KEY_END:
		if (state->arg_num < 1) argp_usage(state);
		break;
	default: return ARGP_ERR_UNKNOWN;
	}
	return 0;
}

static struct argp argp = {options, parse_opt, "sim_file.h5",
                           "DQMC sweep on a B200 GPU, single file version", 0, 0, 0};

int main(int argc, char **argv)
{
	struct arguments a = {0, NULL, false, false, NULL};
	argp_parse(&argp, argc, argv, 0, 0, &a);
	return dqmc_wrapper(a.file, a.log_file, (int64_t)a.time * 1000000000LL, a.dry_run, a.bench);
}
