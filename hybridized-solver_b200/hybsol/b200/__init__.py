"""B200-specific additions: the raw C ABI (``native``), synthetic mesh systems (``meshgen``) and
many independent systems on one device handle (``batch``)."""
