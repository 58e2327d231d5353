#ifndef INCLUDED_CPS_QUDA_H
#define INCLUDED_CPS_QUDA_H
CPS_START_NAMESPACE
class CPSQuda { public: struct QudaParams {}; };
CPS_END_NAMESPACE
#endif
