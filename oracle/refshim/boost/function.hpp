// Test infrastructure only: empty stand-in; the include at fdtd_plrc.t:9 is unused.
