/*
 * dqmc_stack: the job board of the reference's src/main_stack.c, feeding
 * the GPU engine.
 *
 * A stack file lists sim files, one path per line.  Any number of
 * dqmc_stack processes (on any hosts sharing the file system) take jobs from
 * it: a job is popped from the END of the file (LIFO), run, and pushed back
 * to the end if it stopped before finishing (time limit or signal); a job
 * that completes or fails is not pushed back.  The stack file is locked for
 * every pop and push by creating the hard link "<stack>~" (link(2) is
 * atomic); a process that cannot lock retries every 1-3 s, and releases a
 * lock whose modification time has not changed for 10 attempts (its owner
 * is taken to be dead).  A push whose first lock attempt fails first saves
 * the line to "<stack>_<host>_<pid>" so that it survives the process being
 * killed while it waits.  The same semantics as main_stack.c:56-298.
 *
 * Options as the reference (-t max wall seconds for the whole process,
 * -n dry run, -b benchmark mode), plus -k K: pop up to K jobs at a time and
 * run them as chains of one GPU batch (dqmc_wrapper_batch; jobs with equal
 * parameters share kernel launches), pushing back the ones that stopped
 * early.  -k 1 (the default) runs one job at a time through dqmc_wrapper
 * with the log in "<sim file>.log", exactly as the reference does.
 *
 * The environment variable DQMC_STACK_SLEEP scales every sleep (default 1;
 * the tests shorten the waits with it).
 */
#define _GNU_SOURCE
#include <argp.h>
#include <fcntl.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include "dqmc_b200.h"

#define MAX_LEN 512   /* longest path a stack line may hold */

static char host[65];
static int pid;
static double sleep_scale = 1.0;

#define say(...) do { printf("%16s %6d: ", host, pid); printf(__VA_ARGS__); fflush(stdout); } while (0)

static int64_t now_ns(void)
{
	struct timespec t;
	clock_gettime(CLOCK_MONOTONIC, &t);
	return (int64_t)t.tv_sec * 1000000000LL + t.tv_nsec;
}

/* sleep a random time in [lo, hi] seconds, so that processes drift apart */
static void nap(double lo, double hi)
{
	const double t = sleep_scale * (lo + (hi - lo) * (double)rand() / RAND_MAX);
	const struct timespec ts = {(time_t)t, (long)(1e9 * (t - (time_t)t))};
	nanosleep(&ts, NULL);
}

static char *lock_name(const char *file)
{
	const size_t n = strlen(file);
	char *l = malloc(n + 2);
	memcpy(l, file, n);
	l[n] = '~';
	l[n + 1] = 0;
	return l;
}

/* 0 when the lock is taken; with retry == 0, 1 if it is held by another */
static int lock_file(const char *file, int retry)
{
	char *lk = lock_name(file);
	struct timespec last = {0, 0};
	int same = 0;
	for (;;) {
		if (link(file, lk) == 0) {
			free(lk);
			return 0;
		}
		if (!retry) {
			free(lk);
			return 1;
		}
		/* a lock whose mtime stays put for 10 attempts belongs to a dead
		 * process: release it */
		struct stat st;
		if (stat(lk, &st) != 0) {
			same = 0;
		} else if (st.st_mtim.tv_sec == last.tv_sec && st.st_mtim.tv_nsec == last.tv_nsec) {
			same++;
		} else {
			same = 0;
			last = st.st_mtim;
		}
		if (same >= 10) {
			remove(lk);
			say("warning: zombie lock released\n");
			same = 0;
			nap(1.0, 2.0);
		}
		nap(1.0, 3.0);
	}
}

static void unlock_file(const char *file)
{
	char *lk = lock_name(file);
	if (remove(lk) != 0) say("warning: lock release failed (already removed?)\n");
	free(lk);
}

/* Remove the last non-empty line of `file` into `line`: 0 done, 1 the file
 * holds no line (unchanged), -1 an I/O error (unchanged). */
static int pop_stack(const char *file, char *line)
{
	memset(line, 0, MAX_LEN + 1);
	lock_file(file, 1);
	int ret = 0;
	char *buf = NULL;
	const int fd = open(file, O_RDWR);
	if (fd < 0) {
		unlock_file(file);
		say("error: open() failed in pop_stack()\n");
		return -1;
	}
	struct stat st;
	if (fstat(fd, &st) != 0) {
		ret = -1;
		goto out;
	}
	const size_t n = (size_t)st.st_size;
	buf = malloc(n + 1);
	size_t got = 0;
	while (got < n) {
		const ssize_t r = pread(fd, buf + got, n - got, (off_t)got);
		if (r <= 0) break;
		got += (size_t)r;
	}
	if (got != n) {
		say("error: read() failed in pop_stack()\n");
		ret = -1;
		goto out;
	}
	/* the last line: skip trailing newlines and NULs, then back to the
	 * previous newline */
	size_t end = n;
	while (end > 0 && (buf[end - 1] == '\n' || buf[end - 1] == 0)) end--;
	if (end == 0) {
		ret = 1;
		goto out;
	}
	size_t start = end;
	while (start > 0 && buf[start - 1] != '\n') start--;
	if (end - start > MAX_LEN) {
		say("error: last line of %s longer than %d\n", file, MAX_LEN);
		ret = -1;
		goto out;
	}
	memcpy(line, buf + start, end - start);
	if (ftruncate(fd, (off_t)start) != 0) {
		say("error: ftruncate() failed in pop_stack()\n");
		memset(line, 0, MAX_LEN + 1);
		ret = -1;
	}
out:
	free(buf);
	if (close(fd) != 0) say("error: close() failed in pop_stack()\n");
	unlock_file(file);
	return ret;
}

static int append_line(const char *path, const char *line, int create)
{
	const int fd = open(path, O_WRONLY | O_APPEND | (create ? O_CREAT : 0), 0644);
	if (fd < 0) return 1;
	const size_t n = strlen(line);
	int st = 0;
	if (write(fd, line, n) != (ssize_t)n || write(fd, "\n", 1) != 1) st |= 2;
	if (close(fd) != 0) st |= 4;
	return st;
}

/* append `line` to the end of `file` */
static void push_stack(const char *file, const char *line)
{
	char *backup = NULL;
	int st = 0;
	if (lock_file(file, 0) != 0) {
		/* keep the line somewhere while waiting for the lock */
		const size_t n = strlen(file) + 96;
		backup = malloc(n);
		snprintf(backup, n, "%s_%.20s_%d", file, host, pid);
		st |= append_line(backup, line, 1);
		lock_file(file, 1);
	}
	st |= append_line(file, line, 0);
	unlock_file(file);
	if (backup) {
		if (st == 0) remove(backup);
		free(backup);
	}
	if (st & 1) say("error: open() failed in push_stack()\n");
	if (st & 2) say("error: write() failed or incomplete in push_stack()\n");
	if (st & 4) say("error: close() failed in push_stack()\n");
}

static struct argp_option options[] = {
	{0, 't', "TIME", 0, "Max allowed wall time in integer seconds", 0},
	{"dry-run", 'n', 0, 0, "Run through stack, report mem requirement only", 0},
	{"benchmark", 'b', 0, 0, "Don't save sim_data to disk", 0},
	{"batch", 'k', "K", 0, "Jobs popped and run together as one GPU batch (default 1)", 0},
	{0}};

struct arguments {
	int time, batch;
	bool dry, bench;
	char *stack;
};

static error_t parse_opt(int key, char *arg, struct argp_state *state)
{
	struct arguments *a = state->input;
	switch (key) {
	case 't': a->time = atoi(arg); break;
	case 'k': a->batch = atoi(arg); break;
	case 'n': a->dry = true; break;
	case 'b': a->bench = true; break;
	case ARGP_KEY_ARG:
		if (state->arg_num >= 1) argp_usage(state);
		a->stack = arg;
		break;
	case ARGP_KEY_END:
		if (state->arg_num < 1) argp_usage(state);
		break;
	default: return ARGP_ERR_UNKNOWN;
	}
	return 0;
}

static struct argp argp = {options, parse_opt, "stack_file",
                           "DQMC on a B200 GPU, stack version", 0, 0, 0};

int main(int argc, char **argv)
{
	struct arguments a = {0, 1, false, false, NULL};
	argp_parse(&argp, argc, argv, 0, 0, &a);
	if (a.batch < 1) a.batch = 1;
	gethostname(host, 64);
	pid = (int)getpid();
	srand((unsigned)pid);
	const char *sc = getenv("DQMC_STACK_SLEEP");
	if (sc) sleep_scale = atof(sc);
	nap(0.0, 4.0);

	const int64_t t_stop = now_ns() + (int64_t)a.time * 1000000000LL;
	if (access(a.stack, R_OK | W_OK) != 0) {
		say("[ERROR] %s does not exist or you don't have access; idling\n", a.stack);
		return EXIT_FAILURE;
	}
	char (*jobs)[MAX_LEN + 1] = calloc((size_t)a.batch, sizeof(*jobs));
	const char **files = calloc((size_t)a.batch, sizeof(char *));
	int *status = calloc((size_t)a.batch, sizeof(int));
	char log_file[MAX_LEN + 64];
	int ret = EXIT_SUCCESS;
	for (;;) {
		int64_t t_remain = 0;
		if (a.time > 0) {
			t_remain = t_stop - now_ns();
			if (t_remain <= 0) {
				say("dqmc_stack reached wall time limit; idling\n");
				break;
			}
		}
		int n = 0, err = 0;
		while (n < a.batch) {
			const int rc = pop_stack(a.stack, jobs[n]);
			if (rc == -1) { err = 1; break; }
			if (rc == 1) break;
			files[n] = jobs[n];
			n++;
		}
		if (n == 0) {
			if (err) say("[ERROR] pop_stack() failed; idling\n");
			else say("pop_stack() returned 1, %s empty; idling\n", a.stack);
			break;
		}
		int incomplete = 0;
		if (n == 1) {
			snprintf(log_file, sizeof(log_file), "%s.log", files[0]);
			say("starting:   %s\n", files[0]);
			say("logging to: %s\n", log_file);
			status[0] = dqmc_wrapper(files[0], log_file, t_remain, a.dry, a.bench);
		} else {
			snprintf(log_file, sizeof(log_file), "%s_%.20s_%d_batch.log", a.stack, host, pid);
			for (int i = 0; i < n; i++) say("starting:   %s\n", files[i]);
			say("logging to: %s\n", log_file);
			if (a.dry) {
				for (int i = 0; i < n; i++) status[i] = dqmc_wrapper(files[i], log_file, 0, true, false);
			} else {
				dqmc_wrapper_batch(n, files, log_file, t_remain, a.bench, status);
			}
		}
		for (int i = 0; i < n; i++) {
			if (status[i] > 0) {
				push_stack(a.stack, files[i]);
				say("dqmc_wrapper() incomplete, pushed: %s\n", files[i]);
				incomplete = 1;
			} else if (status[i] == 0) {
				say("completed: %s\n", files[i]);
			} else {
				say("dqmc_wrapper() failed: %s\n", files[i]);
			}
		}
		/* a job stops early only on a signal or the time limit */
		if (incomplete) break;
		if (err) {
			say("[ERROR] pop_stack() failed; idling\n");
			break;
		}
	}
	free(jobs);
	free(files);
	free(status);
	return ret;
}
