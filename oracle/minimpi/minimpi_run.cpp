// minimpi_run -n N [-t SECONDS] prog args...
// Starts N ranks of `prog` as forked children connected pairwise by
// socketpairs (see mpi.h). Exits 0 only if every rank exits 0; if one rank
// fails or the optional wall-clock limit passes, the others are killed.
#include <signal.h>
#include <sys/socket.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

int main(int argc, char **argv) {
  int n = 1;
  double limit_s = 0.0;
  int a = 1;
  while (a < argc && argv[a][0] == '-') {
    std::string opt(argv[a]);
    if (opt == "-n" && a + 1 < argc) {
      n = std::atoi(argv[a + 1]);
      a += 2;
    } else if (opt == "-t" && a + 1 < argc) {
      limit_s = std::atof(argv[a + 1]);
      a += 2;
    } else {
      break;
    }
  }
  if (a >= argc || n < 1) {
    std::fprintf(stderr, "usage: minimpi_run -n N [-t SECONDS] prog args...\n");
    return 2;
  }
  std::vector<std::vector<int>> fd((size_t)n, std::vector<int>((size_t)n, -1));
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      int sv[2];
      if (socketpair(AF_UNIX, SOCK_STREAM, 0, sv) != 0) {
        std::perror("socketpair");
        return 2;
      }
      fd[i][j] = sv[0];
      fd[j][i] = sv[1];
    }
  std::vector<pid_t> pids((size_t)n, -1);
  for (int r = 0; r < n; ++r) {
    pid_t p = fork();
    if (p < 0) {
      std::perror("fork");
      return 2;
    }
    if (p == 0) {
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          if (i != r && fd[i][j] >= 0) close(fd[i][j]);
      std::string fds;
      for (int j = 0; j < n; ++j) {
        if (j) fds += ",";
        fds += std::to_string(fd[r][j]);
      }
      setenv("MINIMPI_RANK", std::to_string(r).c_str(), 1);
      setenv("MINIMPI_SIZE", std::to_string(n).c_str(), 1);
      setenv("MINIMPI_FDS", fds.c_str(), 1);
      execvp(argv[a], argv + a);
      std::perror("execvp");
      _exit(127);
    }
    pids[r] = p;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (fd[i][j] >= 0) close(fd[i][j]);

  auto t0 = std::chrono::steady_clock::now();
  int alive = n, rc = 0;
  while (alive > 0) {
    int status = 0;
    pid_t p = waitpid(-1, &status, WNOHANG);
    if (p > 0) {
      --alive;
      int code = WIFEXITED(status) ? WEXITSTATUS(status) : 128 + WTERMSIG(status);
      for (int r = 0; r < n; ++r)
        if (pids[r] == p) pids[r] = -1;
      if (code != 0 && rc == 0) {
        rc = code;
        for (int r = 0; r < n; ++r)
          if (pids[r] > 0) kill(pids[r], SIGKILL);
      }
      continue;
    }
    if (limit_s > 0.0) {
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > limit_s && rc == 0) {
        std::fprintf(stderr, "minimpi_run: wall-clock limit %.0f s reached\n", limit_s);
        rc = 124;
        for (int r = 0; r < n; ++r)
          if (pids[r] > 0) kill(pids[r], SIGKILL);
      }
    }
    std::this_thread::sleep_for(std::chrono::milliseconds(20));
  }
  return rc;
}
