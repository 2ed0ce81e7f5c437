// harness stand-in for glog: logging compiled out
#ifndef REF_STUB_GLOG_H_
#define REF_STUB_GLOG_H_
#endif
