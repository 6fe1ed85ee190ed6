/* driver.c -- filled in below */
#include "case.h"
