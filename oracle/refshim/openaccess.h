/* Oracle build shim (test infrastructure only): included first when the
 * harness is compiled, so that it can reach the reference classes' private
 * members (Core::processdata, Mode's arrays).  The standard headers are
 * pulled in before the access keywords are redefined; the reference objects
 * themselves are compiled unchanged (access does not alter their layout or
 * symbol names). */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>
#include <pthread.h>
#define private public
#define protected public
