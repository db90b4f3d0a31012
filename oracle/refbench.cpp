/*
 * CPU timing of the reference's step_ch() for one configuration.
 * TEST / BASELINE INFRASTRUCTURE ONLY.  Usage: refbench WARM STEPS
 * Prints one JSON object: zones, steps, seconds, zone_cycles_per_s.
 */
#include <stdio.h>
#include <stdlib.h>

extern "C" int ref_init(void);
extern "C" void ref_dims(int *out);
extern "C" double ref_time_steps(int warm, int steps);

int main(int argc, char **argv)
{
  int warm = argc > 1 ? atoi(argv[1]) : 2;
  int steps = argc > 2 ? atoi(argv[2]) : 3;
  int d[16];
  ref_init();
  ref_dims(d);
  double sec = ref_time_steps(warm, steps);
  double zones = (double)d[0] * d[1] * d[2];
  printf("{\"n1\": %d, \"n2\": %d, \"n3\": %d, \"steps\": %d, \"seconds\": %.6f, "
         "\"zone_cycles_per_s\": %.6e}\n", d[0], d[1], d[2], steps, sec, zones * steps / sec);
  return 0;
}
