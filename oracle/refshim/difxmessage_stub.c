/* Oracle build shim (test infrastructure only): the difxmessage calls that
 * the reference's Core, DataStream and alert code make are multicast monitoring only;
 * the oracle drops them. */
#include "difxmessage.h"
int difxMessageInitBinary(void) { return 0; }
int difxMessageSendBinary(const char *data, int destination, int size) { (void)data; (void)destination; (void)size; return 0; }
int difxMessageSendDifxStatus3(enum DifxState state, const char *stateMessage, double visMJD, int numdatastreams, float *weight, double mjdStart, double mjdStop)
{ (void)state; (void)stateMessage; (void)visMJD; (void)numdatastreams; (void)weight; (void)mjdStart; (void)mjdStop; return 0; }
int difxMessageSendDifxAlert(const char *errorMessage, int severity) { (void)errorMessage; (void)severity; return 0; }
int difxMessageSendDifxDiagnosticBufferStatus(int threadid, int numelements, int startelement, int numactiveelements)
{ (void)threadid; (void)numelements; (void)startelement; (void)numactiveelements; return 0; }
int difxMessageSendDifxDiagnosticDataConsumed(long long bytes) { (void)bytes; return 0; }
int difxMessageSendDifxDiagnosticInputDatarate(double bytespersec) { (void)bytespersec; return 0; }
