/* Oracle build shim (test infrastructure only): the difxmessage calls that
 * the reference's Core, DataStream and alert code make are multicast monitoring only;
 * the oracle drops them. */
#include "difxmessage.h"
int difxMessageInitBinary(void) { return 0; }
/* binary messages (STA and kurtosis records) are kept for the harness to read */
static char gx_stub_bin[1 << 22];
static int gx_stub_binlen = 0;
int difxMessageSendBinary(const char *data, int destination, int size)
{
  (void)destination;
  if (size > 0 && gx_stub_binlen + size <= (int)sizeof(gx_stub_bin)) {
    for (int i = 0; i < size; i++) gx_stub_bin[gx_stub_binlen + i] = data[i];
    gx_stub_binlen += size;
  }
  return 0;
}
/* Copies out (at most max bytes of) the kept messages and forgets them. */
int gx_stub_binary_take(char *out, int max)
{
  int n = gx_stub_binlen < max ? gx_stub_binlen : max;
  for (int i = 0; i < n; i++) out[i] = gx_stub_bin[i];
  gx_stub_binlen = 0;
  return n;
}
int difxMessageSendDifxStatus3(enum DifxState state, const char *stateMessage, double visMJD, int numdatastreams, float *weight, double mjdStart, double mjdStop)
{ (void)state; (void)stateMessage; (void)visMJD; (void)numdatastreams; (void)weight; (void)mjdStart; (void)mjdStop; return 0; }
int difxMessageSendDifxAlert(const char *errorMessage, int severity) { (void)errorMessage; (void)severity; return 0; }
int difxMessageSendDifxDiagnosticBufferStatus(int threadid, int numelements, int startelement, int numactiveelements)
{ (void)threadid; (void)numelements; (void)startelement; (void)numactiveelements; return 0; }
int difxMessageSendDifxDiagnosticDataConsumed(long long bytes) { (void)bytes; return 0; }
int difxMessageSendDifxDiagnosticInputDatarate(double bytespersec) { (void)bytespersec; return 0; }
