/* Empty stand-in for <numa.h>: the reference's string headers include it but call no numa_* function. */
#pragma once
