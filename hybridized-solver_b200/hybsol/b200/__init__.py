"""B200-specific additions: the raw C ABI (``native``) and synthetic mesh systems (``meshgen``)."""
