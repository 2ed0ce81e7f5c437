// harness stand-in for chengcli/application's logger: messages are dropped
#ifndef REF_STUB_APPLICATION_HPP_
#define REF_STUB_APPLICATION_HPP_
namespace Application {
struct Logger {
  explicit Logger(const char*) {}
  Logger* operator->() { return this; }
  template <typename... A>
  void Log(A&&...) {}
};
}  // namespace Application
#endif
